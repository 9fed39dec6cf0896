// drtopk_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of Dr.Top-k's selection path (the reference's
// baseline+filter+beta+shuffle radix path, plus the bucket and bitonic
// variants).  It is the checker for the CUDA library: only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.  Nothing in
// drtopksc_b200/ links or calls it.
//
// Parity pins (how this oracle is itself checked):
//   * oracle_radix_final_kth / oracle_bucket_kth / oracle_topk_exact must agree
//     with each other on every input (exactness of the delegate method);
//   * tests/golden/ holds k-th values produced by the reference's own
//     sample_radix_select, compiled from its sources for sm_100a by
//     oracle/Makefile (target ref_harness) and run on a B200 over inputs made
//     by the generators below; tests/test_oracle.py checks this oracle against
//     those fixtures.
//
// Conventions: keys are uint32; "k-th" means the k-th LARGEST (1-based), as in
// the reference (baseline+filter+beta+shuffle/main.cu:286 asserts
// sorted_ascending[N-k] == TopKElement).  Float keys go through the
// order-preserving map of oracle_f32_to_key.

#include <algorithm>
#include <functional>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <thread>
#include <vector>
#include <chrono>

extern "C" {

// ---------------------------------------------------------------- generators
// Seeded streams.  mt19937 output is fixed by the C++ standard, so these are
// reproducible on every machine; normals use our own Box-Muller on mt19937
// words (std::normal_distribution's algorithm is implementation-defined).

void oracle_gen_uniform_u32(uint32_t seed, uint64_t n, uint32_t* out) {
  std::mt19937 g(seed);
  for (uint64_t i = 0; i < n; ++i) out[i] = (uint32_t)g();
}

static inline double u01_open(uint32_t w) { return ((double)w + 0.5) * (1.0 / 4294967296.0); }

static void box_muller(std::mt19937& g, double* z0, double* z1) {
  double u1 = u01_open((uint32_t)g()), u2 = u01_open((uint32_t)g());
  double r = std::sqrt(-2.0 * std::log(u1));
  double t = 6.283185307179586 * u2;
  *z0 = r * std::cos(t);
  *z1 = r * std::sin(t);
}

// clamp(round(N(mean, sd))) to [0, 2^32-1]
void oracle_gen_normal_u32(uint32_t seed, uint64_t n, double mean, double sd, uint32_t* out) {
  std::mt19937 g(seed);
  for (uint64_t i = 0; i < n; i += 2) {
    double z[2];
    box_muller(g, &z[0], &z[1]);
    for (int j = 0; j < 2 && i + j < n; ++j) {
      double v = std::nearbyint(mean + sd * z[j]);
      if (v < 0) v = 0;
      if (v > 4294967295.0) v = 4294967295.0;
      out[i + j] = (uint32_t)v;
    }
  }
}

void oracle_gen_uniform_f32(uint32_t seed, uint64_t n, float* out) {
  std::mt19937 g(seed);
  for (uint64_t i = 0; i < n; ++i) out[i] = (float)((uint32_t)g() >> 8) * (1.0f / 16777216.0f);
}

void oracle_gen_normal_f32(uint32_t seed, uint64_t n, float* out) {
  std::mt19937 g(seed);
  for (uint64_t i = 0; i < n; i += 2) {
    double z[2];
    box_muller(g, &z[0], &z[1]);
    out[i] = (float)z[0];
    if (i + 1 < n) out[i + 1] = (float)z[1];
  }
}

// top 24 bits fixed, low 8 bits uniform: the few-digits / heavy-ties input
void oracle_gen_fewdigits_u32(uint32_t seed, uint64_t n, uint32_t top24, uint32_t* out) {
  std::mt19937 g(seed);
  for (uint64_t i = 0; i < n; ++i) out[i] = (top24 << 8) | ((uint32_t)g() & 0xffu);
}

// Order-preserving float -> uint32 map: negative floats are bit-inverted,
// non-negative ones get the sign bit set.  -0.0 < +0.0; NaNs with the sign
// bit clear sort above +inf, NaNs with it set sort below -inf.
void oracle_f32_to_key(const float* x, uint64_t n, uint32_t* out) {
  for (uint64_t i = 0; i < n; ++i) {
    uint32_t u;
    std::memcpy(&u, &x[i], 4);
    out[i] = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
  }
}

void oracle_key_to_f32(const uint32_t* k, uint64_t n, float* out) {
  for (uint64_t i = 0; i < n; ++i) {
    uint32_t u = (k[i] & 0x80000000u) ? (k[i] & 0x7fffffffu) : ~k[i];
    std::memcpy(&out[i], &u, 4);
  }
}

// ------------------------------------------------------------ alpha / path
// baseline+filter+beta+shuffle/main.cu:83 -- alpha=(int)(0.5*(log2N-log(k)/log(2)+3)),
// evaluated in double exactly as the reference does (the truncation of the
// double result matters when log(k)/log(2) is not exact).
int oracle_ref_alpha(int log2n, double k) {
  int alpha = (int)(0.5 * (log2n - std::log(k) / std::log(2.0) + 3));
  return alpha;
}

// bucket_select/main.cu:66-67 -- same formula, then alpha++ when alpha<5.
int oracle_ref_alpha_bucket(int log2n, double k) {
  int alpha = oracle_ref_alpha(log2n, k);
  if (alpha < 5) alpha++;
  return alpha;
}

// ------------------------------------------------------------ delegates
// baseline+filter+beta+shuffle/radixselect.cuh:882-918 (sampleMax): one max per
// subrange [j*2^alpha, (j+1)*2^alpha) clipped to n; Max starts at 0.
void oracle_sample_max(const uint32_t* x, uint64_t n, int alpha, uint32_t* out) {
  uint64_t S = 1ull << alpha, M = (n + S - 1) / S;
  for (uint64_t j = 0; j < M; ++j) {
    uint32_t m = 0;
    uint64_t e = std::min(n, (j + 1) * S);
    for (uint64_t i = j * S; i < e; ++i) m = std::max(m, x[i]);
    out[j] = m;
  }
}

// radixselect.cuh:966-1041 (sampleMax_NoReduction_Beta2): Max=first key,
// Second=0, ascending scan "if Max<v {Second=Max;Max=v} else if Second<v
// {Second=v}".  out[2j]=Max, out[2j+1]=Second.  With >=2 keys per subrange
// Second is the multiset second-largest.
void oracle_sample_top2(const uint32_t* x, uint64_t n, int alpha, uint32_t* out) {
  uint64_t S = 1ull << alpha, M = (n + S - 1) / S;
  for (uint64_t j = 0; j < M; ++j) {
    uint64_t b = j * S, e = std::min(n, (j + 1) * S);
    uint32_t mx = x[b], sc = 0;
    for (uint64_t i = b + 1; i < e; ++i) {
      uint32_t v = x[i];
      if (mx < v) { sc = mx; mx = v; }
      else if (sc < v) sc = v;
    }
    out[2 * j] = mx;
    out[2 * j + 1] = sc;
  }
}

// ------------------------------------------------------------ digit select
static inline uint32_t prefix_of(uint32_t v, int shleft) {
  // CUDA's shr/shl clamp shift amounts >= 32 to a result of 0; the reference
  // relies on that for the first digit (shleft = 32 matches every key).
  return shleft >= 32 ? 0u : ((v >> shleft) << shleft);
}

// One MSD radix-select run over v[0..n) with the reference's host digit loop
// (radixselect.cuh:1410-1470 radix_select_inplace, 1666-1724 _firsttopk,
// 1727-1780 _firsttopk_beta) and CumulateCount_inplace (191-220): for each
// digit, histogram the keys whose higher digits equal flag's
// (CalculateOccurence_inplace, 352-410), accumulate ascending from Belowcount
// and take the smallest bin with CumCount >= n-k+1.
//   start_digit: first digit processed (32/nbits-1 in the reference)
//   stop_digit : loop runs while digit >= stop_digit (0 = all; 3 = beta path)
//   early_stop : break after a digit whose chosen bin holds one key (_firsttopk)
// Returns flag; *out_digit receives the digit index after the loop (so the
// reference's follow-up shleft is (*out_digit+1)*nbits).
uint32_t oracle_digit_select(const uint32_t* v, uint64_t n, int64_t k, int nbits,
                             int start_digit, int stop_digit, int early_stop, int* out_digit) {
  const int B = 1 << nbits;
  std::vector<int64_t> cnt(B), cum(B);
  uint32_t flag = 0;
  int64_t below = 0;
  const int64_t target = (int64_t)n - k + 1;
  int cur = start_digit;
  while (cur >= stop_digit) {
    int shleft = (cur + 1) * nbits, shright = cur * nbits;
    std::fill(cnt.begin(), cnt.end(), 0);
    for (uint64_t i = 0; i < n; ++i)
      if (prefix_of(v[i], shleft) == flag) cnt[(v[i] >> shright) & (uint32_t)(B - 1)]++;
    int64_t sum = below;
    int kd = 0;
    for (int i = 0; i < B; ++i) {
      sum += cnt[i];
      cum[i] = sum;
      bool hit = (i == 0) ? (cum[0] >= target) : (cum[i] >= target && cum[i - 1] < target);
      if (hit) { kd = i; flag |= (uint32_t)i << shright; }
    }
    if (kd != 0) below = cum[kd - 1];
    int64_t kcount = cnt[kd];
    cur--;
    if (early_stop && kcount == 1) break;
  }
  if (out_digit) *out_digit = cur;
  return flag;
}

typedef struct {
  int alpha, beta_path;        // beta_path: 1 when the top-2 (beta=2) path ran
  uint64_t n_subranges;        // M
  uint32_t first_flag;         // threshold from the first select
  int first_digits;            // digits the first select processed
  uint64_t n_selected;         // subranges whose keys were concatenated
  uint64_t n_lonely;           // elements appended by the lonely rule (beta path)
  uint64_t n_candidates;       // size of the concatenated vector
} oracle_stats;

// Full FINAL path: sample_radix_select, radixselect.cuh:1782-1894, for the
// beta=1 ("default", alpha>5) and beta=2 (alpha<=5) branches.
//   FindTopKRanges 412-427 + FillWithKElementsID 602-618: subranges with
//   prefix > flag, topped up with prefix == flag ones to exactly k.  The
//   reference tops up with whichever ids win its atomics; this restatement
//   takes the lowest ids (the k-th value does not depend on the choice).
//   FindTopKRanges_beta 560-598: Max>=flag && Second>=flag -> subrange
//   selected; Max>=flag only -> (Max, Second) appended as lonely elements.
//   CreateConcatenateRange_(Beta_)optimized 1574-1639: keys >= flag.
//   Second select: radix_select_inplace over all digits (1888-1891).
// Returns 0 on success, -1 on invalid input (k<1, k>n, nbits not in
// {1,2,4,8}, or the default path with fewer than k subranges).
int oracle_radix_final_kth(const uint32_t* x, uint64_t n, int64_t k, int nbits, int alpha,
                           int force_path, uint32_t* kth, oracle_stats* st) {
  if (k < 1 || (uint64_t)k > n) return -1;
  if (!(nbits == 1 || nbits == 2 || nbits == 4 || nbits == 8)) return -1;
  const int D = 32 / nbits;
  oracle_stats s;
  std::memset(&s, 0, sizeof(s));
  s.alpha = alpha;
  if (alpha == 0) {  // main.cu:253-258: plain radix_select
    int d;
    *kth = oracle_digit_select(x, n, k, nbits, D - 1, 0, 0, &d);
    s.first_digits = D;
    s.n_candidates = n;
    if (st) *st = s;
    return 0;
  }
  // main.cu:87-89 -- defaultContribution = alpha > 5; force_path 1/2 overrides
  int beta_path = (force_path == 0) ? (alpha <= 5) : (force_path == 2);
  s.beta_path = beta_path;
  uint64_t S = 1ull << alpha, M = (n + S - 1) / S;
  s.n_subranges = M;
  std::vector<uint32_t> cand;
  if (!beta_path) {
    if (M < (uint64_t)k) return -1;
    std::vector<uint32_t> del(M);
    oracle_sample_max(x, n, alpha, del.data());
    int d;
    uint32_t flag = oracle_digit_select(del.data(), M, k, nbits, D - 1, 0, 1, &d);
    int shleft = (d + 1) * nbits;
    s.first_flag = flag;
    s.first_digits = (D - 1) - d;
    std::vector<uint64_t> sel;
    for (uint64_t j = 0; j < M; ++j)
      if (prefix_of(del[j], shleft) > flag) sel.push_back(j);
    for (uint64_t j = 0; j < M && sel.size() < (uint64_t)k; ++j)
      if (prefix_of(del[j], shleft) == flag) sel.push_back(j);
    s.n_selected = sel.size();
    for (uint64_t j : sel) {
      uint64_t e = std::min(n, (j + 1) * S);
      for (uint64_t i = j * S; i < e; ++i)
        if (x[i] >= flag) cand.push_back(x[i]);
    }
  } else {
    std::vector<uint32_t> del(2 * M);
    oracle_sample_top2(x, n, alpha, del.data());
    int d;
    // radix_select_inplace_firsttopk_beta: while(CurrentDigit>=3), no early stop
    uint32_t flag = oracle_digit_select(del.data(), 2 * M, k, nbits, D - 1, 3, 0, &d);
    s.first_flag = flag;
    s.first_digits = (D - 1) - d;
    std::vector<uint64_t> sel;
    for (uint64_t j = 0; j < M; ++j) {
      uint32_t mx = del[2 * j], sc = del[2 * j + 1];
      if (mx >= flag) {
        if (sc >= flag) sel.push_back(j);
        else { cand.push_back(mx); cand.push_back(sc); s.n_lonely += 2; }
      }
    }
    s.n_selected = sel.size();
    for (uint64_t j : sel) {
      uint64_t e = std::min(n, (j + 1) * S);
      for (uint64_t i = j * S; i < e; ++i)
        if (x[i] >= flag) cand.push_back(x[i]);
    }
  }
  s.n_candidates = cand.size();
  int d;
  *kth = oracle_digit_select(cand.data(), cand.size(), k, nbits, D - 1, 0, 0, &d);
  if (st) *st = s;
  return 0;
}

// ------------------------------------------------------------ exact top-k
// The top-level oracle: the Enabletest check of main.cu:281-296 (kth ==
// ascending[N-k]) extended to the full top-k: every index whose key is > kth,
// then the lowest indices whose key == kth, sorted by key descending then
// index ascending.  vals/idx may be NULL.
void oracle_topk_exact(const uint32_t* x, uint64_t n, int64_t k, uint32_t* kth, uint32_t* vals,
                       int64_t* idx) {
  std::vector<uint32_t> tmp(x, x + n);
  std::nth_element(tmp.begin(), tmp.begin() + (n - k), tmp.end());
  uint32_t K = tmp[n - k];
  *kth = K;
  if (!vals && !idx) return;
  std::vector<std::pair<uint32_t, uint64_t>> out;
  out.reserve(k);
  uint64_t gt = 0;
  for (uint64_t i = 0; i < n; ++i) gt += (x[i] > K);
  uint64_t need_eq = (uint64_t)k - gt;
  for (uint64_t i = 0; i < n; ++i) {
    if (x[i] > K) out.push_back({x[i], i});
    else if (x[i] == K && need_eq) { out.push_back({x[i], i}); need_eq--; }
  }
  std::sort(out.begin(), out.end(), [](const std::pair<uint32_t, uint64_t>& a,
                                       const std::pair<uint32_t, uint64_t>& b) {
    return a.first != b.first ? a.first > b.first : a.second < b.second;
  });
  for (int64_t i = 0; i < k; ++i) {
    if (vals) vals[i] = out[i].first;
    if (idx) idx[i] = (int64_t)out[i].second;
  }
}

// Multi-threaded host top-k (the CPU baseline): each of T threads copies its
// slice and keeps its top k with nth_element, the T*k survivors are reduced
// with one more nth_element, and the top k are sorted descending.  Returns
// wall seconds (copy included, data generation excluded).
double oracle_topk_mt(const uint32_t* x, uint64_t n, int64_t k, int threads, uint32_t* kth,
                      uint32_t* vals) {
  auto t0 = std::chrono::steady_clock::now();
  if (threads < 1) threads = 1;
  std::vector<std::vector<uint32_t>> part(threads);
  std::vector<std::thread> th;
  for (int t = 0; t < threads; ++t) {
    th.emplace_back([&, t]() {
      uint64_t b = n * t / threads, e = n * (t + 1) / threads;
      std::vector<uint32_t> w(x + b, x + e);
      uint64_t kk = std::min<uint64_t>((uint64_t)k, w.size());
      if (kk < w.size())
        std::nth_element(w.begin(), w.begin() + kk, w.end(), std::greater<uint32_t>());
      w.resize(kk);
      part[t].swap(w);
    });
  }
  for (auto& t : th) t.join();
  std::vector<uint32_t> all;
  for (auto& p : part) all.insert(all.end(), p.begin(), p.end());
  std::nth_element(all.begin(), all.begin() + (k - 1), all.end(), std::greater<uint32_t>());
  *kth = all[k - 1];
  std::sort(all.begin(), all.begin() + k, std::greater<uint32_t>());
  if (vals) std::memcpy(vals, all.data(), sizeof(uint32_t) * k);
  auto t1 = std::chrono::steady_clock::now();
  return std::chrono::duration<double>(t1 - t0).count();
}

// ------------------------------------------------------------ bucket variant
// Integer-exact restatement of the Dr.Top-k bucket select
// (bucket_select/bucketselect_combined.cuh): the reference computes bucket
// ids as (int)((v-min)*slope) in double and returns "any key of the final
// bucket" (GetKValue, 270-298), which is not exact.  Here a bucket over the
// inclusive range [lo,hi] with nb buckets has integer width
// w = (hi-lo)/nb + 1 and bucket(v) = (v-lo)/w.
//
// bucket_refine: select over keys in [lo,hi] with remaining rank R (counted
// from the top inside the range).  Each level picks the highest bucket b
// whose suffix count reaches R, narrows the range to bucket b, and subtracts
// the keys above it.  Stops when the range is one value, when the chosen
// bucket holds one key (stop_on_single), or after max_levels levels.
// Returns the final range lower bound; *exact receives the k-th value when
// the select finished (single key or single value), else is left unchanged.
static uint32_t bucket_refine(const uint32_t* v, uint64_t n, uint32_t lo, uint32_t hi, int64_t R,
                              int nb, int max_levels, int stop_on_single, uint32_t* exact,
                              int* levels_done) {
  std::vector<int64_t> cnt(nb);
  int lv = 0;
  while (lo < hi && lv < max_levels) {
    uint64_t w = (uint64_t)(hi - lo) / (uint64_t)nb + 1;
    std::fill(cnt.begin(), cnt.end(), 0);
    for (uint64_t i = 0; i < n; ++i)
      if (v[i] >= lo && v[i] <= hi) cnt[(uint64_t)(v[i] - lo) / w]++;
    int64_t suf = 0;
    int b = 0;
    for (int i = nb - 1; i >= 0; --i) {
      if (suf + cnt[i] >= R) { b = i; break; }
      suf += cnt[i];
    }
    R -= suf;
    uint64_t nlo = (uint64_t)lo + (uint64_t)b * w;
    uint64_t nhi = std::min<uint64_t>(hi, nlo + w - 1);
    lo = (uint32_t)nlo;
    hi = (uint32_t)nhi;
    lv++;
    if (stop_on_single && cnt[b] == 1) {
      for (uint64_t i = 0; i < n; ++i)
        if (v[i] >= lo && v[i] <= hi) { *exact = v[i]; break; }
      if (levels_done) *levels_done = lv;
      return lo;
    }
  }
  if (lo == hi) *exact = lo;
  if (levels_done) *levels_done = lv;
  return lo;
}

// Exact bucket select of the k-th largest of v (bucket_select 472-568 +
// bucket_select_PhaseII 349-470, integer buckets): min/max, then refine.
uint32_t oracle_bucket_select(const uint32_t* v, uint64_t n, int64_t k, int nb) {
  uint32_t lo = 0xffffffffu, hi = 0;
  for (uint64_t i = 0; i < n; ++i) { lo = std::min(lo, v[i]); hi = std::max(hi, v[i]); }
  uint32_t ex = lo;
  bucket_refine(v, n, lo, hi, k, nb, 1 << 30, 1, &ex, nullptr);
  return ex;
}

// Full Dr.Top-k bucket path (sample_bucket_select 1279-1358):
//   default path (alpha>5): first select refines to the exact k-th delegate
//   D (bucket_select_inplaceFirstTopk 1131-1276), selects subranges with
//   delegate > D topped up with == D (lowest ids), gathers keys >= D;
//   beta path: two bucket levels on the (Max,Second) delegates
//   (bucket_select_inplace_betaFirstTopk 972-1095), threshold = lower bound of
//   the final bucket, lonely rule as in the radix path.
int oracle_bucket_kth(const uint32_t* x, uint64_t n, int64_t k, int nb, int alpha, int force_path,
                      uint32_t* kth, oracle_stats* st) {
  if (k < 1 || (uint64_t)k > n || nb < 2) return -1;
  oracle_stats s;
  std::memset(&s, 0, sizeof(s));
  s.alpha = alpha;
  int beta_path = (force_path == 0) ? (alpha <= 5) : (force_path == 2);
  s.beta_path = beta_path;
  uint64_t S = 1ull << alpha, M = (n + S - 1) / S;
  s.n_subranges = M;
  std::vector<uint32_t> cand;
  if (!beta_path) {
    if (M < (uint64_t)k) return -1;
    std::vector<uint32_t> del(M);
    oracle_sample_max(x, n, alpha, del.data());
    uint32_t D = oracle_bucket_select(del.data(), M, k, nb);
    s.first_flag = D;
    uint64_t nsel = 0;
    std::vector<uint64_t> sel;
    for (uint64_t j = 0; j < M; ++j) if (del[j] > D) sel.push_back(j);
    for (uint64_t j = 0; j < M && sel.size() < (uint64_t)k; ++j) if (del[j] == D) sel.push_back(j);
    nsel = sel.size();
    s.n_selected = nsel;
    for (uint64_t j : sel) {
      uint64_t e = std::min(n, (j + 1) * S);
      for (uint64_t i = j * S; i < e; ++i) if (x[i] >= D) cand.push_back(x[i]);
    }
  } else {
    std::vector<uint32_t> del(2 * M);
    oracle_sample_top2(x, n, alpha, del.data());
    uint32_t lo = 0xffffffffu, hi = 0;
    for (uint64_t i = 0; i < 2 * M; ++i) { lo = std::min(lo, del[i]); hi = std::max(hi, del[i]); }
    uint32_t ex = 0;
    int lv = 0;
    uint32_t T = (2 * M >= (uint64_t)k) ? bucket_refine(del.data(), 2 * M, lo, hi, k, nb, 2, 0, &ex, &lv) : 0u;
    s.first_flag = T;
    s.first_digits = lv;
    uint64_t nsel = 0;
    for (uint64_t j = 0; j < M; ++j) {
      uint32_t mx = del[2 * j], sc = del[2 * j + 1];
      if (mx >= T) {
        if (sc >= T) {
          nsel++;
          uint64_t e = std::min(n, (j + 1) * S);
          for (uint64_t i = j * S; i < e; ++i) if (x[i] >= T) cand.push_back(x[i]);
        } else { cand.push_back(mx); cand.push_back(sc); s.n_lonely += 2; }
      }
    }
    s.n_selected = nsel;
  }
  s.n_candidates = cand.size();
  *kth = oracle_bucket_select(cand.data(), cand.size(), k, nb);
  if (st) *st = s;
  return 0;
}

// ------------------------------------------------------------ bitonic variant
// Dr.Top-k bitonic (bitonic/bitonic_com.cuh 609-728): the k subranges with the
// largest delegates (ties: lowest id) are concatenated whole, and the sorted
// top-k of that concatenation is the answer.  Restated with a plain sort;
// the network itself is the GPU's business.  Requires M >= k.
int oracle_bitonic_topk(const uint32_t* x, uint64_t n, int64_t k, int alpha, uint32_t* vals,
                        int64_t* idx) {
  uint64_t S = 1ull << alpha, M = (n + S - 1) / S;
  if (k < 1 || M < (uint64_t)k) return -1;
  std::vector<uint32_t> del(M);
  oracle_sample_max(x, n, alpha, del.data());
  std::vector<uint64_t> ids(M);
  for (uint64_t j = 0; j < M; ++j) ids[j] = j;
  std::partial_sort(ids.begin(), ids.begin() + k, ids.end(), [&](uint64_t a, uint64_t b) {
    return del[a] != del[b] ? del[a] > del[b] : a < b;
  });
  std::vector<std::pair<uint32_t, uint64_t>> c;
  for (int64_t t = 0; t < k; ++t) {
    uint64_t j = ids[t], e = std::min(n, (j + 1) * S);
    for (uint64_t i = j * S; i < e; ++i) c.push_back({x[i], i});
  }
  std::partial_sort(c.begin(), c.begin() + k, c.end(),
                    [](const std::pair<uint32_t, uint64_t>& a, const std::pair<uint32_t, uint64_t>& b) {
                      return a.first != b.first ? a.first > b.first : a.second < b.second;
                    });
  for (int64_t i = 0; i < k; ++i) {
    if (vals) vals[i] = c[i].first;
    if (idx) idx[i] = (int64_t)c[i].second;
  }
  return 0;
}

// BMW experiment (BMW/radixselect.cuh:1746-1832 with the min-heap of
// BMW/PQ.h): one delegate (Max) per subrange of 2^alpha keys, then one
// sequential scan that keeps the k largest keys seen in a min-heap; once the
// heap holds k keys its minimum is the threshold, a key enters only above it
// (evicting the minimum), and a subrange whose Max is below the threshold is
// skipped whole.  The reference makes the heap's minimum the threshold from
// the first push on, so while the heap is not yet full it can drop keys the
// answer needs; here the threshold applies once the heap is full, which
// keeps the k-th exact.  Returns the k-th largest key; *skipped counts the
// keys never examined.
uint32_t oracle_bmw_kth(const uint32_t* x, uint64_t n, int64_t k, int alpha, uint64_t* skipped) {
  const uint64_t S = 1ull << alpha, M = (n + S - 1) / S;
  std::vector<uint32_t> del(M);
  oracle_sample_max(x, n, alpha, del.data());
  std::vector<uint32_t> heap;  // min-heap
  heap.reserve((size_t)k + 1);
  auto gt = std::greater<uint32_t>();
  uint64_t skip = 0;
  for (uint64_t j = 0; j < M; ++j) {
    const uint64_t b = j * S, e = std::min(n, b + S);
    const bool full = heap.size() == (size_t)k;
    if (full && del[j] < heap.front()) {
      skip += e - b;
      continue;
    }
    for (uint64_t i = b; i < e; ++i) {
      if (heap.size() < (size_t)k) {
        heap.push_back(x[i]);
        std::push_heap(heap.begin(), heap.end(), gt);
      } else if (x[i] > heap.front()) {
        std::pop_heap(heap.begin(), heap.end(), gt);
        heap.back() = x[i];
        std::push_heap(heap.begin(), heap.end(), gt);
      }
    }
  }
  if (skipped) *skipped = skip;
  return heap.front();
}

// FNV-1a over the sorted top-k (values then indices): a compact fixture digest.
uint64_t oracle_digest(const uint32_t* vals, const int64_t* idx, int64_t k) {
  uint64_t h = 1469598103934665603ull;
  for (int64_t i = 0; i < k; ++i) {
    uint32_t v = vals[i];
    for (int b = 0; b < 4; ++b) { h ^= (v >> (8 * b)) & 0xff; h *= 1099511628211ull; }
  }
  if (idx)
    for (int64_t i = 0; i < k; ++i) {
      uint64_t v = (uint64_t)idx[i];
      for (int b = 0; b < 8; ++b) { h ^= (v >> (8 * b)) & 0xff; h *= 1099511628211ull; }
    }
  return h;
}

}  // extern "C"
