// ref_harness.cu -- TEST INFRASTRUCTURE ONLY (builds oracle/_ref/ref_harness).
//
// Runs the reference's own Dr.Top-k radix select -- sample_radix_select from
// baseline+filter+beta+shuffle/radixselect.cuh, #included from the read-only
// reference tree at build time, never copied -- over inputs made by the
// seeded generators of drtopk_oracle.cpp, so that its k-th values and stage
// counters can be committed as golden fixtures and its B200 timings measured
// beside ours.
//
// Buffer set-up follows baseline+filter+beta+shuffle/main.cu:140-250 (alpha
// formula, scratch sizes, launch constants, the caller zeroing the two
// counters before each call); only the data source differs (seeded instead
// of std::random_device).  Buffers are sized once for the largest request of
// a k list, so one process serves a whole sweep over one generated input.
//
// usage:
//   ref_harness <dist> <log2n> <k[,k...]> <nbits> <beta> <seed> [reps]
//       one line  RESULT {json}  per k on stdout: the k-th value, alpha/path,
//       the reference's counters (CountSelectedSubrange, CountLonelyElements,
//       write_pos) and its stage times.
//   ref_harness --bench <dist> <log2n> <k,k,...> <nbits> <beta> <seed> <steps> <warmup> <e2e_steps>
//       times the stock call over the k list: `steps` sweeps with the keys
//       resident (CUDA events around each sweep), then `e2e_steps` sweeps that
//       also upload the keys from pinned host memory before every call; one
//       line  BENCH {json}.
//   dist: u32 | normal | fewdigits | f32u | f32n
// The reference's own chatter goes to stderr.

#include "radixselect.cuh"

#include <cstdint>
#include <cstdio>
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
  std::fflush(stdout);
  return 2;
}

static bool gen_keys(const std::string& dist, uint32_t seed, uint64_t n, uint32_t* out) {
  if (dist == "u32") oracle_gen_uniform_u32(seed, n, out);
  else if (dist == "normal") oracle_gen_normal_u32(seed, n, 2147483648.0, 268435456.0, out);
  else if (dist == "fewdigits") oracle_gen_fewdigits_u32(seed, n, 0xABCDEFu, out);
  else if (dist == "f32u" || dist == "f32n") {
    std::vector<float> f(n);
    if (dist == "f32u") oracle_gen_uniform_f32(seed, n, f.data());
    else oracle_gen_normal_f32(seed, n, f.data());
    oracle_f32_to_key(f.data(), n, out);
  } else return false;
  return true;
}

// main.cu:83-92 and 215-225: the parameters of one call
struct RefCfg {
  int k, alpha, SubRangesize, NSubranges, NthreadstoworkInreduction;
  bool defaultContribution;
  int NThreadsPerBlock, SizeOfSubWarp, pow_size_Subwarp, NSharedMemoryElements, SizeOfAllocation;
  int NSubRangesPerBlock, NSubWarps_InBlock, NElementsPerBlock_ReadFromGlobal, TotalBlocksrequired;
  const char* refusal;  // non-null: the harness does not run this k (reason)
};

static RefCfg make_cfg(int log2n, int k) {
  RefCfg c;
  std::memset(&c, 0, sizeof(c));
  const int num_element = 1 << log2n;
  c.k = k;
  c.alpha = 0.5 * (log2n - log(k) / log(2) + 3);
  c.defaultContribution = !(c.alpha <= 5);
  c.SubRangesize = pow(2, c.alpha);
  c.NSubranges = num_element / c.SubRangesize;
  c.NthreadstoworkInreduction = c.SubRangesize < 32 ? c.SubRangesize : 32;
  c.NThreadsPerBlock = 256;
  c.SizeOfSubWarp = 8;
  c.pow_size_Subwarp = 3;
  c.NSharedMemoryElements = c.NThreadsPerBlock << 5;
  c.SizeOfAllocation = c.NSharedMemoryElements + (c.NSharedMemoryElements >> 5);
  c.NSubRangesPerBlock = c.NSharedMemoryElements / c.SizeOfSubWarp;
  c.NSubWarps_InBlock = c.NThreadsPerBlock >> c.pow_size_Subwarp;
  c.NElementsPerBlock_ReadFromGlobal = c.NSubRangesPerBlock * c.SubRangesize;
  c.TotalBlocksrequired = num_element / c.NElementsPerBlock_ReadFromGlobal;
  // Inputs the reference does not handle (checked before any launch): the
  // default path reads k selected ids, so it needs NSubranges >= k; the
  // staged beta sampler reads 256*2^alpha keys per block unguarded.
  if (k < 1 || k > num_element) c.refusal = "k out of range";
  else if (c.alpha == 0) c.refusal = "alpha==0 (plain radix) not exercised by the harness";
  else if (c.defaultContribution && c.NSubranges < k) c.refusal = "NSubranges < k on the default path";
  else if (!c.defaultContribution && (num_element % (256 << c.alpha)) != 0)
    c.refusal = "N not a multiple of 256*2^alpha";
  else if (c.TotalBlocksrequired < 1) c.refusal = "TotalBlocksrequired < 1";
  return c;
}

struct RefBufs {
  data_t* vec_d = nullptr;
  data_t* Max_d = nullptr;
  index_t* SubrangeId_d = nullptr;
  index_t *SelectedSubrangeId_d = nullptr, *CountSelectedSubrange_d = nullptr, *CountLonelyElements_d = nullptr,
          *write_pos_d = nullptr;
  data_t* ConcatenatedRange_d = nullptr;
};

// main.cu:205-250: scratch sized for the largest delegate vector of the list
static void alloc_bufs(RefBufs& b, int num_element, long max_delegates) {
  H_ERR(cudaMalloc((void**)&b.vec_d, sizeof(data_t) * num_element));
  H_ERR(cudaMalloc((void**)&b.Max_d, sizeof(data_t) * max_delegates));
  H_ERR(cudaMalloc((void**)&b.SubrangeId_d, sizeof(index_t) * max_delegates));
  H_ERR(cudaMalloc((void**)&b.SelectedSubrangeId_d, sizeof(index_t) * num_element));
  H_ERR(cudaMalloc((void**)&b.CountSelectedSubrange_d, sizeof(index_t)));
  H_ERR(cudaMalloc((void**)&b.CountLonelyElements_d, sizeof(index_t)));
  H_ERR(cudaMalloc((void**)&b.ConcatenatedRange_d, sizeof(data_t) * num_element));
  H_ERR(cudaMalloc((void**)&b.write_pos_d, sizeof(index_t)));
}

struct CallOut {
  data_t kth;
  double tS, tF, t2, tC;
};

// one stock call, preceded by the caller's counter zeroing (main.cu:243-244)
static CallOut ref_call(RefBufs& b, int num_element, int NBits, int beta, const RefCfg& c) {
  H_ERR(cudaMemset(b.CountSelectedSubrange_d, 0, sizeof(index_t)));
  H_ERR(cudaMemset(b.CountLonelyElements_d, 0, sizeof(index_t)));
  const int num_bucket = 1 << NBits;
  const int CurrentDigit = (32 / NBits) - 1;
  CallOut o;
  o.kth = 0;
  o.tS = o.tF = o.t2 = o.tC = 0;
  sample_radix_select<data_t, index_t>(b.vec_d, num_element, c.k, num_bucket, o.kth, NBits, CurrentDigit,
      c.NSubranges, c.SubRangesize, c.alpha, o.tS, o.tF, o.t2, o.tC, b.Max_d, b.SubrangeId_d,
      c.NSharedMemoryElements, c.SizeOfSubWarp, c.pow_size_Subwarp, c.NSubWarps_InBlock, c.NSubRangesPerBlock,
      c.NElementsPerBlock_ReadFromGlobal, c.TotalBlocksrequired, c.SizeOfAllocation, c.NThreadsPerBlock, beta,
      c.defaultContribution, c.NthreadstoworkInreduction, b.SelectedSubrangeId_d, b.CountLonelyElements_d,
      b.write_pos_d, b.ConcatenatedRange_d, b.CountSelectedSubrange_d);
  return o;
}

static std::vector<int> parse_ks(const char* s) {
  std::vector<int> ks;
  const char* p = s;
  while (*p) {
    ks.push_back(std::atoi(p));
    while (*p && *p != ',') ++p;
    if (*p == ',') ++p;
  }
  return ks;
}

static int run_fixtures(int argc, char** argv) {
  if (argc < 7) return fail("usage: ref_harness dist log2n k[,k...] nbits beta seed [reps]");
  std::string dist = argv[1];
  int log2n = std::atoi(argv[2]);
  std::vector<int> ks = parse_ks(argv[3]);
  int NBits = std::atoi(argv[4]);
  int beta = std::atoi(argv[5]);
  uint32_t seed = (uint32_t)std::strtoul(argv[6], nullptr, 10);
  int reps = argc > 7 ? std::atoi(argv[7]) : 1;
  if (log2n < 10 || log2n > 30) return fail("log2n must be in [10,30]");
  if (!(NBits == 1 || NBits == 2 || NBits == 4 || NBits == 8)) return fail("nbits must be 1,2,4,8");
  if (beta != 2) return fail("only beta=2 is valid in the reference (beta 3/4 paths are buggy)");
  if (ks.empty()) return fail("no k");
  const int num_element = 1 << log2n;

  std::vector<RefCfg> cfgs;
  long max_del = 1;
  for (int k : ks) {
    RefCfg c = make_cfg(log2n, k);
    cfgs.push_back(c);
    if (!c.refusal) max_del = std::max<long>(max_del, (long)c.NSubranges * beta);
  }
  std::vector<uint32_t> vec(num_element);
  if (!gen_keys(dist, seed, num_element, vec.data())) return fail("unknown dist");

  RefBufs b;
  alloc_bufs(b, num_element, max_del);
  H_ERR(cudaMemcpy(b.vec_d, vec.data(), sizeof(data_t) * num_element, cudaMemcpyHostToDevice));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  for (const RefCfg& c : cfgs) {
    if (c.refusal) {
      std::printf("RESULT {\"dist\": \"%s\", \"log2n\": %d, \"k\": %d, \"nbits\": %d, \"seed\": %u, "
                  "\"error\": \"%s\"}\n", dist.c_str(), log2n, c.k, NBits, seed, c.refusal);
      std::fflush(stdout);
      continue;
    }
    data_t first_kth = 0;
    index_t cnt_sel = 0, cnt_lonely = 0, wpos = 0;
    double best_ms = 1e30, best_wall = 1e30, t_s = 0, t_f = 0, t_c = 0, t_2 = 0;
    bool changed = false;
    for (int r = 0; r < reps; ++r) {
      H_ERR(cudaDeviceSynchronize());
      double w0 = wtime();
      cudaEventRecord(e0);
      CallOut o = ref_call(b, num_element, NBits, beta, c);
      cudaEventRecord(e1);
      cudaEventSynchronize(e1);
      double wall = (wtime() - w0) * 1e3;
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      if (r == 0) {
        first_kth = o.kth;
        // the reference's observable counters after its first call
        H_ERR(cudaMemcpy(&cnt_sel, b.CountSelectedSubrange_d, sizeof(index_t), cudaMemcpyDeviceToHost));
        H_ERR(cudaMemcpy(&cnt_lonely, b.CountLonelyElements_d, sizeof(index_t), cudaMemcpyDeviceToHost));
        H_ERR(cudaMemcpy(&wpos, b.write_pos_d, sizeof(index_t), cudaMemcpyDeviceToHost));
      }
      if (o.kth != first_kth) changed = true;
      if (wall < best_wall) {
        best_wall = wall;
        best_ms = ms;
        t_s = o.tS * 1e3; t_f = o.tF * 1e3; t_c = o.tC * 1e3; t_2 = o.t2 * 1e3;
      }
    }
    if (changed) return fail("k-th value changed between repetitions");
    std::printf(
        "RESULT {\"dist\": \"%s\", \"log2n\": %d, \"k\": %d, \"nbits\": %d, \"beta\": %d, "
        "\"seed\": %u, \"alpha\": %d, \"path\": \"%s\", \"kth\": %u, \"count_selected\": %d, "
        "\"count_lonely\": %d, \"write_pos\": %d, \"reps\": %d, "
        "\"ms_event\": %.4f, \"ms_wall\": %.4f, \"ms_sample\": %.4f, \"ms_first\": %.4f, "
        "\"ms_concat\": %.4f, \"ms_second\": %.4f}\n",
        dist.c_str(), log2n, c.k, NBits, beta, seed, c.alpha, c.defaultContribution ? "D" : "B",
        (unsigned)first_kth, cnt_sel, cnt_lonely, wpos, reps, best_ms, best_wall, t_s, t_f, t_c, t_2);
    std::fflush(stdout);
  }
  return 0;
}

static int run_bench(int argc, char** argv) {
  // argv: --bench dist log2n ks nbits beta seed steps warmup e2e_steps
  if (argc < 11) return fail("usage: ref_harness --bench dist log2n k,k,... nbits beta seed steps warmup e2e_steps");
  std::string dist = argv[2];
  int log2n = std::atoi(argv[3]);
  std::vector<int> ks = parse_ks(argv[4]);
  int NBits = std::atoi(argv[5]);
  int beta = std::atoi(argv[6]);
  uint32_t seed = (uint32_t)std::strtoul(argv[7], nullptr, 10);
  int steps = std::atoi(argv[8]), warmup = std::atoi(argv[9]), e2e_steps = std::atoi(argv[10]);
  if (log2n < 10 || log2n > 30) return fail("log2n must be in [10,30]");
  if (!(NBits == 1 || NBits == 2 || NBits == 4 || NBits == 8) || beta != 2) return fail("nbits 1,2,4,8 and beta 2");
  if (ks.empty() || steps < 1) return fail("no k or no steps");
  const int num_element = 1 << log2n;
  std::vector<RefCfg> cfgs;
  long max_del = 1;
  for (int k : ks) {
    RefCfg c = make_cfg(log2n, k);
    if (c.refusal) return fail(c.refusal);
    cfgs.push_back(c);
    max_del = std::max<long>(max_del, (long)c.NSubranges * beta);
  }
  uint32_t* host = nullptr;  // pinned, as a caller streaming its keys would hold them
  H_ERR(cudaMallocHost((void**)&host, sizeof(uint32_t) * (size_t)num_element));
  if (!gen_keys(dist, seed, num_element, host)) return fail("unknown dist");
  RefBufs b;
  alloc_bufs(b, num_element, max_del);
  H_ERR(cudaMemcpy(b.vec_d, host, sizeof(data_t) * num_element, cudaMemcpyHostToDevice));
  std::vector<data_t> kth(cfgs.size(), 0);
  std::vector<double> per_k_ms(cfgs.size(), 0.0);
  cudaEvent_t e0, e1, a0, a1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventCreate(&a0);
  cudaEventCreate(&a1);
  for (int w = 0; w < warmup; ++w)
    for (size_t i = 0; i < cfgs.size(); ++i) kth[i] = ref_call(b, num_element, NBits, beta, cfgs[i]).kth;
  H_ERR(cudaDeviceSynchronize());
  // resident keys: CUDA events around each sweep; per-k events inside it
  double total_ms = 0;
  for (int s = 0; s < steps; ++s) {
    cudaEventRecord(e0);
    for (size_t i = 0; i < cfgs.size(); ++i) {
      cudaEventRecord(a0);
      data_t v = ref_call(b, num_element, NBits, beta, cfgs[i]).kth;
      cudaEventRecord(a1);
      cudaEventSynchronize(a1);
      float ms = 0;
      cudaEventElapsedTime(&ms, a0, a1);
      per_k_ms[i] += ms;
      if (v != kth[i]) return fail("k-th value changed between calls");
    }
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    total_ms += ms;
  }
  // end to end: the keys are uploaded from pinned memory before every call
  double e2e_ms = 0;
  for (int s = 0; s < e2e_steps; ++s) {
    cudaEventRecord(e0);
    for (size_t i = 0; i < cfgs.size(); ++i) {
      H_ERR(cudaMemcpy(b.vec_d, host, sizeof(data_t) * num_element, cudaMemcpyHostToDevice));
      data_t v = ref_call(b, num_element, NBits, beta, cfgs[i]).kth;
      if (v != kth[i]) return fail("k-th value changed between calls");
    }
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    e2e_ms += ms;
  }
  std::printf("BENCH {\"dist\": \"%s\", \"log2n\": %d, \"nbits\": %d, \"beta\": %d, \"seed\": %u, \"steps\": %d, "
              "\"warmup\": %d, \"e2e_steps\": %d, \"ms_total\": %.4f, \"e2e_ms_total\": %.4f, \"per_k\": [",
              dist.c_str(), log2n, NBits, beta, seed, steps, warmup, e2e_steps, total_ms, e2e_ms);
  for (size_t i = 0; i < cfgs.size(); ++i)
    std::printf("%s{\"k\": %d, \"alpha\": %d, \"path\": \"%s\", \"kth\": %u, \"ms\": %.4f}", i ? ", " : "",
                cfgs[i].k, cfgs[i].alpha, cfgs[i].defaultContribution ? "D" : "B", (unsigned)kth[i],
                per_k_ms[i] / steps);
  std::printf("]}\n");
  std::fflush(stdout);
  return 0;
}

int main(int argc, char** argv) {
  // Send the reference's cout chatter to stderr so stdout carries results only.
  std::cout.rdbuf(std::cerr.rdbuf());
  if (argc > 1 && std::string(argv[1]) == "--bench") return run_bench(argc, argv);
  return run_fixtures(argc, argv);
}
