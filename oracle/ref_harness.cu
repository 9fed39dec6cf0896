// ref_harness.cu -- TEST INFRASTRUCTURE ONLY (builds oracle/_ref/ref_harness).
//
// Runs the reference's own Dr.Top-k radix select -- sample_radix_select from
// baseline+filter+beta+shuffle/radixselect.cuh, #included from the read-only
// reference tree at build time, never copied -- over inputs made by the
// seeded generators of drtopk_oracle.cpp, so that its k-th values can be
// committed as golden fixtures and its B200 timings reported beside ours.
//
// Buffer set-up follows baseline+filter+beta+shuffle/main.cu:140-250 (alpha
// formula, scratch sizes, launch constants); only the data source differs
// (seeded instead of std::random_device).
//
// usage: ref_harness <dist> <log2n> <k> <nbits> <beta> <seed> [reps]
//   dist: u32 | normal | fewdigits | f32u | f32n
// prints one line  RESULT {json}  on stdout (the reference's own chatter is
// sent to stderr).

#include "radixselect.cuh"

#include <cstdio>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

// main.cu:14-15 -- the reference's key and index types
typedef unsigned int data_t;
typedef int index_t;

extern "C" {
void oracle_gen_uniform_u32(uint32_t seed, uint64_t n, uint32_t* out);
void oracle_gen_normal_u32(uint32_t seed, uint64_t n, double mean, double sd, uint32_t* out);
void oracle_gen_uniform_f32(uint32_t seed, uint64_t n, float* out);
void oracle_gen_normal_f32(uint32_t seed, uint64_t n, float* out);
void oracle_gen_fewdigits_u32(uint32_t seed, uint64_t n, uint32_t top24, uint32_t* out);
void oracle_f32_to_key(const float* x, uint64_t n, uint32_t* out);
}

static int fail(const char* m) {
  std::printf("RESULT {\"error\": \"%s\"}\n", m);
  return 2;
}

int main(int argc, char** argv) {
  if (argc < 7) return fail("usage: ref_harness dist log2n k nbits beta seed [reps]");
  std::string dist = argv[1];
  int log2n = std::atoi(argv[2]);
  int k = std::atoi(argv[3]);
  int NBits = std::atoi(argv[4]);
  int beta = std::atoi(argv[5]);
  uint32_t seed = (uint32_t)std::strtoul(argv[6], nullptr, 10);
  int reps = argc > 7 ? std::atoi(argv[7]) : 1;
  if (log2n < 10 || log2n > 30) return fail("log2n must be in [10,30]");
  int num_element = 1 << log2n;
  if (k < 1 || k > num_element) return fail("k out of range");
  if (!(NBits == 1 || NBits == 2 || NBits == 4 || NBits == 8)) return fail("nbits must be 1,2,4,8");
  if (beta != 2) return fail("only beta=2 is valid in the reference (beta 3/4 paths are buggy)");

  // Send the reference's cout chatter to stderr so stdout carries RESULT only.
  std::cout.rdbuf(std::cerr.rdbuf());

  std::vector<uint32_t> vec(num_element);
  if (dist == "u32") oracle_gen_uniform_u32(seed, num_element, vec.data());
  else if (dist == "normal") oracle_gen_normal_u32(seed, num_element, 2147483648.0, 268435456.0, vec.data());
  else if (dist == "fewdigits") oracle_gen_fewdigits_u32(seed, num_element, 0xABCDEFu, vec.data());
  else if (dist == "f32u" || dist == "f32n") {
    std::vector<float> f(num_element);
    if (dist == "f32u") oracle_gen_uniform_f32(seed, num_element, f.data());
    else oracle_gen_normal_f32(seed, num_element, f.data());
    oracle_f32_to_key(f.data(), num_element, vec.data());
  } else return fail("unknown dist");

  // main.cu:83-92
  int alpha = 0.5 * (log2n - log(k) / log(2) + 3);
  bool defaultContribution = !(alpha <= 5);
  int SubRangesize = pow(2, alpha);
  int num_bucket = 1 << NBits;
  int CurrentDigit = (32 / NBits) - 1;
  int NSubranges = num_element / SubRangesize;
  int NthreadstoworkInreduction = SubRangesize < 32 ? SubRangesize : 32;
  // main.cu:215-225 launch constants of the staged beta sampler
  int NThreadsPerBlock = 256, SizeOfSubWarp = 8, pow_size_Subwarp = 3;
  int NSharedMemoryElements = NThreadsPerBlock << 5;
  int SizeOfAllocation = NSharedMemoryElements + (NSharedMemoryElements >> 5);
  int NSubRangesPerBlock = NSharedMemoryElements / SizeOfSubWarp;
  int NSubWarps_InBlock = NThreadsPerBlock >> pow_size_Subwarp;
  int NElementsPerBlock_ReadFromGlobal = NSubRangesPerBlock * SubRangesize;
  int TotalBlocksrequired = num_element / NElementsPerBlock_ReadFromGlobal;

  // Guards for inputs the reference does not handle (checked before any
  // launch): the default path reads k selected ids, so it needs NSubranges>=k;
  // the staged beta sampler reads 256*2^alpha keys per block unguarded.
  if (alpha == 0) return fail("alpha==0 (plain radix) not exercised by the harness");
  if (defaultContribution && NSubranges < k) return fail("NSubranges < k on the default path");
  if (!defaultContribution && (num_element % (256 << alpha)) != 0) return fail("N not a multiple of 256*2^alpha");
  if (TotalBlocksrequired < 1) return fail("TotalBlocksrequired < 1");

  data_t* vec_d;
  H_ERR(cudaMalloc((void**)&vec_d, sizeof(data_t) * num_element));
  H_ERR(cudaMemcpy(vec_d, vec.data(), sizeof(data_t) * num_element, cudaMemcpyHostToDevice));
  data_t* Max_d;
  index_t* SubrangeId_d;
  H_ERR(cudaMalloc((void**)&Max_d, sizeof(data_t) * NSubranges * beta));
  H_ERR(cudaMalloc((void**)&SubrangeId_d, sizeof(index_t) * NSubranges * beta));
  index_t *SelectedSubrangeId_d, *CountSelectedSubrange_d, *CountLonelyElements_d, *write_pos_d;
  data_t* ConcatenatedRange_d;
  H_ERR(cudaMalloc((void**)&SelectedSubrangeId_d, sizeof(index_t) * num_element));
  H_ERR(cudaMalloc((void**)&CountSelectedSubrange_d, sizeof(index_t)));
  H_ERR(cudaMalloc((void**)&CountLonelyElements_d, sizeof(index_t)));
  H_ERR(cudaMalloc((void**)&ConcatenatedRange_d, sizeof(data_t) * num_element));
  H_ERR(cudaMalloc((void**)&write_pos_d, sizeof(index_t)));

  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  data_t first_kth = 0;
  double best_ms = 1e30, t_s = 0, t_f = 0, t_c = 0, t_2 = 0, best_wall = 1e30;
  for (int r = 0; r < reps; ++r) {
    // main.cu:243-244: the two counters are zeroed by the caller before a call
    H_ERR(cudaMemset(CountSelectedSubrange_d, 0, sizeof(index_t)));
    H_ERR(cudaMemset(CountLonelyElements_d, 0, sizeof(index_t)));
    H_ERR(cudaDeviceSynchronize());
    data_t TopKElement = 0;
    double tS = 0, tF = 0, t2 = 0, tC = 0;
    double w0 = wtime();
    cudaEventRecord(e0);
    sample_radix_select<data_t, index_t>(vec_d, num_element, k, num_bucket, TopKElement, NBits,
        CurrentDigit, NSubranges, SubRangesize, alpha, tS, tF, t2, tC, Max_d, SubrangeId_d,
        NSharedMemoryElements, SizeOfSubWarp, pow_size_Subwarp, NSubWarps_InBlock,
        NSubRangesPerBlock, NElementsPerBlock_ReadFromGlobal, TotalBlocksrequired,
        SizeOfAllocation, NThreadsPerBlock, beta, defaultContribution, NthreadstoworkInreduction,
        SelectedSubrangeId_d, CountLonelyElements_d, write_pos_d, ConcatenatedRange_d,
        CountSelectedSubrange_d);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    double wall = (wtime() - w0) * 1e3;
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r == 0) first_kth = TopKElement;
    if (TopKElement != first_kth) return fail("k-th value changed between repetitions");
    if (wall < best_wall) {
      best_wall = wall;
      best_ms = ms;
      t_s = tS * 1e3; t_f = tF * 1e3; t_c = tC * 1e3; t_2 = t2 * 1e3;
    }
  }
  std::printf(
      "RESULT {\"dist\": \"%s\", \"log2n\": %d, \"k\": %d, \"nbits\": %d, \"beta\": %d, "
      "\"seed\": %u, \"alpha\": %d, \"path\": \"%s\", \"kth\": %u, \"reps\": %d, "
      "\"ms_event\": %.4f, \"ms_wall\": %.4f, \"ms_sample\": %.4f, \"ms_first\": %.4f, "
      "\"ms_concat\": %.4f, \"ms_second\": %.4f}\n",
      dist.c_str(), log2n, k, NBits, beta, seed, alpha, defaultContribution ? "D" : "B",
      (unsigned)first_kth, reps, best_ms, best_wall, t_s, t_f, t_c, t_2);
  std::fflush(stdout);
  return 0;
}
