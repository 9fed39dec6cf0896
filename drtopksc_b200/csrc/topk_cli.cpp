// topk_cli.cpp -- drop-in for the reference's topk.bin
// (baseline+filter+beta+shuffle/main.cu:56-323): same positional argv
// "log2N k NBitsPerDigit beta", same result lines, same CSV row
// "D|B; log2N;k;alpha;beta;sample;first;concat;second;normal;total" (ms).
// The data are uniform uint32 from a seeded mt19937 (the reference uses an
// unseeded random_device); --seed S, --dist u32|normal|fewdigits|f32u|f32n,
// --algo radix|bucket|plain, --alpha A, --csv FILE, --check are extras.
//
// The real-dataset build (RealDatasets/BinaryDataset/main.cu:56-148) takes
// "log2N k NBitsPerDigit beta scoreFile output_file": with six positional
// arguments the keys come from scoreFile and the CSV row goes to
// output_file.  --format txt (default: the reference's default build, "%f"
// scores and its unsigned arithmetic), bin (raw int32, the readBinary build)
// or score ((1 - s) * 1e9 in float) picks the reader (drtopk_load_dataset);
// --input FILE does the same with the four-argument form.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <random>
#include <string>
#include <vector>
#include <algorithm>

#include "drtopk.h"

static void gen(const std::string& dist, uint32_t seed, std::vector<uint32_t>& v) {
  std::mt19937 g(seed);
  const size_t n = v.size();
  if (dist == "u32") {
    for (size_t i = 0; i < n; ++i) v[i] = (uint32_t)g();
  } else if (dist == "fewdigits") {
    for (size_t i = 0; i < n; ++i) v[i] = (0xABCDEFu << 8) | ((uint32_t)g() & 0xffu);
  } else {
    for (size_t i = 0; i < n; i += 2) {
      double u1 = ((double)(uint32_t)g() + 0.5) / 4294967296.0, u2 = ((double)(uint32_t)g() + 0.5) / 4294967296.0;
      double r = std::sqrt(-2.0 * std::log(u1)), t = 6.283185307179586 * u2;
      double z[2] = {r * std::cos(t), r * std::sin(t)};
      for (int j = 0; j < 2 && i + j < n; ++j) {
        if (dist == "normal") {
          double x = std::nearbyint(2147483648.0 + 268435456.0 * z[j]);
          x = std::min(4294967295.0, std::max(0.0, x));
          v[i + j] = (uint32_t)x;
        } else {
          float f = (float)z[j];
          std::memcpy(&v[i + j], &f, 4);
        }
      }
    }
    if (dist == "f32u")
      for (size_t i = 0; i < n; ++i) {
        float f = (float)((uint32_t)g() >> 8) * (1.0f / 16777216.0f);
        std::memcpy(&v[i], &f, 4);
      }
  }
}

int main(int argc, char** argv) {
  std::printf("./exe num_element k NBitsPerDigit beta\n");
  std::vector<std::string> pos;
  uint32_t seed = 1;
  std::string dist = "u32", algo = "radix", csv = "drtopk_b200.csv", input, format = "txt";
  int alpha_opt = -1;
  bool check = false;
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    if (a == "--seed" && i + 1 < argc) seed = (uint32_t)std::strtoul(argv[++i], nullptr, 10);
    else if (a == "--dist" && i + 1 < argc) dist = argv[++i];
    else if (a == "--algo" && i + 1 < argc) algo = argv[++i];
    else if (a == "--alpha" && i + 1 < argc) alpha_opt = std::atoi(argv[++i]);
    else if (a == "--csv" && i + 1 < argc) csv = argv[++i];
    else if (a == "--check") check = true;
    else if (a == "--input" && i + 1 < argc) input = argv[++i];
    else if (a == "--format" && i + 1 < argc) format = argv[++i];
    else pos.push_back(a);
  }
  if (pos.size() == 6) {  // RealDatasets/BinaryDataset/main.cu:58-59: ... scoreFile output_file
    input = pos[4];
    csv = pos[5];
    pos.resize(4);
  }
  if (pos.size() != 4) { std::printf("wrong input\n"); return 1; }
  int fmt = -1;
  if (!input.empty()) {
    fmt = format == "bin" ? DRTOPK_DATASET_BIN_I32
                          : (format == "txt" ? DRTOPK_DATASET_TXT_REF
                                             : (format == "score" ? DRTOPK_DATASET_TXT_SCORE : -1));
    if (fmt < 0) { std::printf("wrong input\n"); return 1; }
  }
  const int log2n = std::atoi(pos[0].c_str());
  const long long k = std::atoll(pos[1].c_str());
  const int nbits = std::atoi(pos[2].c_str());
  const int beta = std::atoi(pos[3].c_str());
  if (log2n < 1 || log2n > 31) { std::printf("wrong input\n"); return 1; }
  const uint64_t n = 1ull << log2n;
  std::printf("num_element: %llu\n", (unsigned long long)n);
  std::vector<uint32_t> h(n);
  if (!input.empty()) {
    uint64_t got = 0;
    if (drtopk_load_dataset(input.c_str(), fmt, n, h.data(), &got) != DRTOPK_OK) {
      std::printf("Error! opening SCORE file\n");
      return 1;
    }
    dist = "u32";  // dataset keys are uint32
    std::printf("read %llu values from %s\n", (unsigned long long)got, input.c_str());
  } else {
    gen(dist, seed, h);
  }
  drtopk_params_t p;
  drtopk_params_default(&p);
  p.nbits = nbits;
  p.beta = beta;
  p.alpha = alpha_opt;
  if (algo == "bucket") { p.algo = DRTOPK_ALGO_BUCKET; p.num_bucket = 1 << nbits; }
  else if (algo == "plain") p.algo = DRTOPK_ALGO_PLAIN_RADIX;
  const drtopk_dtype_t dt = (dist == "f32u" || dist == "f32n") ? DRTOPK_F32 : DRTOPK_U32;
  void* d = nullptr;
  uint32_t* dk = nullptr;
  if (cudaMalloc(&d, n * 4) != cudaSuccess || cudaMalloc(&dk, 4) != cudaSuccess) { std::printf("cudaMalloc failed\n"); return 2; }
  cudaMemcpy(d, h.data(), n * 4, cudaMemcpyHostToDevice);
  drtopk_handle_t H;
  if (drtopk_create(&H, 0, 0) != DRTOPK_OK) { std::printf("drtopk_create failed\n"); return 2; }
  // one untimed call sizes the resident workspace (the reference allocates scratch before its timer too)
  drtopk_status_t s = drtopk_select(H, d, dt, n, (uint64_t)k, &p, dk, nullptr, nullptr, nullptr);
  if (s == DRTOPK_OK) s = drtopk_sync_check(H, nullptr);
  if (s != DRTOPK_OK) { std::printf("drtopk_select failed: %s\n", drtopk_status_str(s)); return 3; }
  auto t0 = std::chrono::steady_clock::now();
  s = drtopk_select(H, d, dt, n, (uint64_t)k, &p, dk, nullptr, nullptr, nullptr);
  if (s == DRTOPK_OK) s = drtopk_sync_check(H, nullptr);
  auto t1 = std::chrono::steady_clock::now();
  if (s != DRTOPK_OK) { std::printf("drtopk_select failed: %s\n", drtopk_status_str(s)); return 3; }
  uint32_t kth = 0;
  cudaMemcpy(&kth, dk, 4, cudaMemcpyDeviceToHost);
  drtopk_stats_t st;
  drtopk_last_stats(H, &st);
  const double total = std::chrono::duration<double, std::milli>(t1 - t0).count();
  std::printf("Calculated alpha: %d\n", st.alpha);
  if (dt == DRTOPK_F32) { float f; std::memcpy(&f, &kth, 4); std::printf("The kth element from top is:%.9g\n", f); }
  else std::printf("The kth element from top is:%u\n", kth);
  std::printf("Sampling Time:%g ms\n", st.ms_sample);
  std::printf("Time for First TopK:%g ms\n", st.ms_first);
  std::printf("Time for Concatenation:%g ms\n", st.ms_concat);
  std::printf("Time for Second TopK:%g ms\n", st.ms_second);
  std::printf("Time for Normal Radix Select:%g ms\n", st.beta == 0 ? st.ms_total : 0.0);
  std::printf("Total Time:%g ms\n", total);
  int rc = 0;
  if (check) {
    std::vector<uint32_t> c(h);
    if (dt == DRTOPK_F32)
      for (auto& u : c) u = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
    std::nth_element(c.begin(), c.begin() + (n - k), c.end());
    uint32_t want = c[n - k];
    if (dt == DRTOPK_F32) want = (want & 0x80000000u) ? (want & 0x7fffffffu) : ~want;
    std::printf(want == kth ? "Success!\n" : "Not Success!\n");
    std::printf("Required value%u\n", want);
    rc = want == kth ? 0 : 4;
  }
  std::ofstream f(csv, std::ios::app);
  f << (st.beta == 2 ? "B" : "D") << "; " << log2n << ";" << k << ";" << st.alpha << ";" << beta << ";" << st.ms_sample
    << ";" << st.ms_first << ";" << st.ms_concat << ";" << st.ms_second << ";" << (st.beta == 0 ? st.ms_total : 0.0)
    << ";" << total << "\n";
  drtopk_destroy(H);
  cudaFree(d);
  cudaFree(dk);
  return rc;
}
