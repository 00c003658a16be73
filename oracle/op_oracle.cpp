// CPU oracle for finpar/OptionPricing.fut (entry main, f32) -- TEST
// INFRASTRUCTURE ONLY.  It is the checker of the GPU pricer and the timed CPU
// baseline; no product path links or calls it.
//
// Each Monte-Carlo path is restated step by step from the reference, in f32
// with one IEEE rounding per operation in the reference's order (the library
// is built with -ffp-contract=off):
//   Sobol point of path n (1-based) from the Gray code of n   :13-33
//   inverse Gaussian (Wichura's AS241 rational approximations) :36-136
//   Brownian bridge per underlying                             :142-175
//   correlation (lower-triangular) and prices (exp, product scan) :188-228
//   the three contracts' payoffs                               :234-301
//   mean over paths per model                                  :304-322
// Two choices the reference leaves open are fixed here, identically in the
// GPU kernels: f32.exp and f32.log are taken as the f32 rounding of the f64
// function (within half an f32 ulp of the exact value, where f32 library
// versions differ by an ulp between platforms), and the sum over paths -- a
// `reduce` whose order the reference does not specify -- is accumulated in
// f64 and rounded to f32 before the division by num_mc_it.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace {

struct OpArgs {
  int contract, num_mc_it, num_bits, num_models, num_und, num_dates, num_discts;
  const int32_t* dir_vs;     // [num_dates * num_und][num_bits]
  const float* md_cs;        // [num_models][num_und][num_und]
  const float* md_vols;      // [num_models][num_dates][num_und]
  const float* md_drifts;    // [num_models][num_dates][num_und]
  const float* md_sts;       // [num_models][num_und]
  const float* md_detvals;   // [num_models][1]
  const float* md_discts;    // [num_models][num_discts]
  const int32_t* bb_inds;    // [3][num_dates]
  const float* bb_data;      // [3][num_dates]
};

inline float f32exp(float x) { return (float)std::exp((double)x); }
inline float f32log(float x) { return (float)std::log((double)x); }

// :52-57
inline float poly_appr(float x, const float* a, const float* b) {
  const float num = x * (x * (x * (x * (x * (x * (x * a[7] + a[6]) + a[5]) + a[4]) + a[3]) + a[2]) + a[1]) + a[0];
  const float den = x * (x * (x * (x * (x * (x * (x * b[7] + b[6]) + b[5]) + b[4]) + b[3]) + b[2]) + b[1]) + b[0];
  return num / den;
}

// The coefficient tables of :59-118 (AS241, Wichura 1988), as f32 literals.
const float kSmallA[8] = {3.387132872796366608f, 133.14166789178437745f, 1971.5909503065514427f,
                          13731.693765509461125f, 45921.953931549871457f, 67265.770927008700853f,
                          33430.575583588128105f, 2509.0809287301226727f};
const float kSmallB[8] = {1.0f, 42.313330701600911252f, 687.1870074920579083f, 5394.1960214247511077f,
                          21213.794301586595867f, 39307.89580009271061f, 28729.085735721942674f,
                          5226.495278852854561f};
const float kInterA[8] = {1.42343711074968357734f, 4.6303378461565452959f, 5.7694972214606914055f,
                          3.64784832476320460504f, 1.27045825245236838258f, 0.24178072517745061177f,
                          0.0227238449892691845833f, 7.7454501427834140764e-4f};
const float kInterB[8] = {1.0f, 2.05319162663775882187f, 1.6763848301838038494f, 0.68976733498510000455f,
                          0.14810397642748007459f, 0.0151986665636164571966f, 5.475938084995344946e-4f,
                          1.05075007164441684324e-9f};
const float kTailA[8] = {6.6579046435011037772f, 5.4637849111641143699f, 1.7848265399172913358f,
                         0.29656057182850489123f, 0.026532189526576123093f, 0.0012426609473880784386f,
                         2.71155556874348757815e-5f, 2.01033439929228813265e-7f};
const float kTailB[8] = {1.0f, 0.59983220655588793769f, 0.13692988092273580531f, 0.0148753612908506148525f,
                         7.868691311456132591e-4f, 1.8463183175100546818e-5f, 1.4215117583164458887e-7f,
                         2.04426310338993978564e-5f};

// :120-136
inline float ugaussian_el(float p) {
  const float dp = p - 0.5f;
  if ((dp < 0.0f && 0.0f - dp <= 0.425f) || (0.0f <= dp && dp <= 0.425f))
    return dp * poly_appr(0.180625f - dp * dp, kSmallA, kSmallB);
  const float pp = dp < 0.0f ? dp + 0.5f : 0.5f - dp;
  const float r = std::sqrt(-f32log(pp));
  const float x = r <= 5.0f ? poly_appr(r - 1.6f, kInterA, kInterB) : poly_appr(r - 5.0f, kTailA, kTailB);
  return dp < 0.0f ? 0.0f - x : x;
}

// :234-240
inline float fmin_payoff(const float* xs) {
  const float a = xs[0] / 3758.05f, b = xs[1] / 11840.0f, c = xs[2] / 1200.0f;
  return a < b ? (a < c ? a : c) : (b < c ? b : c);
}

// One path's payoff under every model, added to acc[num_models].
void op_path(const OpArgs& q, int32_t n, float* gauss, float* bbrow, float* bb, float* prices, double* acc) {
  const int D = q.num_dates, U = q.num_und, K = D * U, B = q.num_bits;
  // Sobol point (:13-33) and inverse Gaussian: gauss[d][u]
  const int32_t gray = (n >> 1) ^ n;
  const float divisor = std::pow(2.0f, (float)B);
  for (int k = 0; k < K; k++) {
    int32_t x = 0;
    for (int i = 0; i < B; i++) {
      const int32_t t = (int32_t)((uint32_t)1 << i);
      if ((gray & t) == t) x ^= q.dir_vs[(int64_t)k * B + i];
    }
    gauss[k] = ugaussian_el((float)x / divisor);
  }
  // Brownian bridge per underlying (:142-175): bb[d][u]
  const int32_t* bi = q.bb_inds;
  const int32_t* li = q.bb_inds + D;
  const int32_t* ri = q.bb_inds + 2 * D;
  const float* sd = q.bb_data;
  const float* lw = q.bb_data + D;
  const float* rw = q.bb_data + 2 * D;
  for (int u = 0; u < U; u++) {
    for (int d = 0; d < D; d++) bbrow[d] = 0.0f;
    bbrow[bi[0] - 1] = sd[0] * gauss[0 * U + u];
    for (int i = 1; i < D; i++) {
      const int j = li[i] - 1, k = ri[i] - 1, l = bi[i] - 1;
      const float wk = bbrow[k];
      const float zi = gauss[i * U + u];
      const float tmp = rw[i] * wk + sd[i] * zi;
      bbrow[l] = j == -1 ? tmp : tmp + lw[i] * bbrow[j];
    }
    for (int ii = 1; ii < D; ii++) {
      const int i = D - ii;
      bbrow[i] = bbrow[i] - bbrow[i - 1];
    }
    for (int d = 0; d < D; d++) bb[d * U + u] = bbrow[d];
  }
  for (int m = 0; m < q.num_models; m++) {
    const float* c = q.md_cs + (int64_t)m * U * U;
    const float* vols = q.md_vols + (int64_t)m * D * U;
    const float* drifts = q.md_drifts + (int64_t)m * D * U;
    const float* starts = q.md_sts + (int64_t)m * U;
    // correlateDeltas (:188-199), combineVs and mkPrices (:201-218)
    for (int u = 0; u < U; u++) {
      float acc_scan = 1.0f;
      for (int d = 0; d < D; d++) {
        float noise = 0.0f;
        for (int i = 0; i <= u; i++) noise = noise + bb[d * U + i] * c[u * U + i];
        const float cv = drifts[d * U + u] + noise * vols[d * U + u];
        acc_scan = acc_scan * f32exp(cv);
        prices[d * U + u] = starts[u] * acc_scan;
      }
    }
    // payoffs (:242-301)
    const float* disc = q.md_discts + (int64_t)m * q.num_discts;
    float pay = 0.0f;
    if (q.contract == 1) {
      const float amount = (prices[0] - 4000.0f) * q.md_detvals[m];
      const float amount0 = 0.0f < amount ? amount : 0.0f;
      pay = amount0 * disc[0];
    } else if (q.contract == 2) {
      int date;
      float amount;
      if (1.0f <= fmin_payoff(prices + 0 * 3)) date = 0, amount = 1150.0f;
      else if (1.0f <= fmin_payoff(prices + 1 * 3)) date = 1, amount = 1300.0f;
      else if (1.0f <= fmin_payoff(prices + 2 * 3)) date = 2, amount = 1450.0f;
      else if (1.0f <= fmin_payoff(prices + 3 * 3)) date = 3, amount = 1600.0f;
      else {
        const float x50 = fmin_payoff(prices + 4 * 3);
        date = 4;
        amount = 1.0f <= x50 ? 1750.0f : (0.75f < x50 ? 1000.0f : x50 * 1000.0f);
      }
      pay = amount * disc[date];
    } else if (q.contract == 3) {
      bool cond = false;
      for (int d = 0; d < 367; d++) {
        const float* x = prices + d * 3;
        cond = cond || (x[0] <= 2630.6349999999998f || x[1] <= 8288.0f || x[2] <= 840.0f);
      }
      const float price1 = 100.0f * disc[0];
      const float* last = prices + 366 * 3;
      const bool goto40 = cond && (last[0] < 3758.05f || last[1] < 11840.0f || last[2] < 1200.0f);
      const float amount = goto40 ? 1000.0f * fmin_payoff(last) : 1000.0f;
      const float price2 = amount * disc[1];
      pay = price1 + price2;
    }
    acc[m] += (double)pay;
  }
}

}  // namespace

extern "C" {

// The contract's required (num_dates, num_und): (1, 1), (5, 3), (367, 3); 0
// when the shapes fit, else 1 (the reference's size coercion fails).
int lvc_oracle_op_shape_ok(int contract, int num_dates, int num_und) {
  if (contract == 1) return num_dates == 1 && num_und == 1 ? 0 : 1;
  if (contract == 2) return num_dates == 5 && num_und == 3 ? 0 : 1;
  if (contract == 3) return num_dates == 367 && num_und == 3 ? 0 : 1;
  return 0;
}

// main of finpar/OptionPricing.fut on paths [first, first + count) (1-based
// Sobol indices first + 1 ...), their payoff sums per model into sums[] (f64,
// summed in path order within each of `threads` contiguous ranges, then the
// ranges in order).  num_discts >= 2 for contract 3, >= 5 for contract 2.
void lvc_oracle_op_sums(int contract, int num_bits, int num_models, int num_und, int num_dates, int num_discts,
                        const int32_t* dir_vs, const float* md_cs, const float* md_vols, const float* md_drifts,
                        const float* md_sts, const float* md_detvals, const float* md_discts, const int32_t* bb_inds,
                        const float* bb_data, int64_t first, int64_t count, int threads, double* sums) {
  OpArgs q{contract, 0, num_bits, num_models, num_und, num_dates, num_discts, dir_vs, md_cs, md_vols, md_drifts,
           md_sts, md_detvals, md_discts, bb_inds, bb_data};
  if (threads < 1) threads = 1;
  std::vector<std::vector<double>> part(threads, std::vector<double>(num_models, 0.0));
  auto work = [&](int t) {
    const int64_t lo = first + count * t / threads, hi = first + count * (t + 1) / threads;
    const int K = num_dates * num_und;
    std::vector<float> gauss(K), bbrow(num_dates), bb(K), prices(K);
    for (int64_t it = lo; it < hi; it++)
      op_path(q, (int32_t)(it + 1), gauss.data(), bbrow.data(), bb.data(), prices.data(), part[t].data());
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < threads; t++) pool.emplace_back(work, t);
  work(0);
  for (auto& th : pool) th.join();
  for (int m = 0; m < num_models; m++) {
    double s = 0.0;
    for (int t = 0; t < threads; t++) s += part[t][m];
    sums[m] = s;
  }
}

// The f32 payoffs of paths [first, first + count), [path][model] -- for
// checks of how the reference's reduce over paths may have been ordered.
void lvc_oracle_op_payoffs(int contract, int num_bits, int num_models, int num_und, int num_dates, int num_discts,
                           const int32_t* dir_vs, const float* md_cs, const float* md_vols, const float* md_drifts,
                           const float* md_sts, const float* md_detvals, const float* md_discts,
                           const int32_t* bb_inds, const float* bb_data, int64_t first, int64_t count, int threads,
                           float* out) {
  OpArgs q{contract, 0, num_bits, num_models, num_und, num_dates, num_discts, dir_vs, md_cs, md_vols, md_drifts,
           md_sts, md_detvals, md_discts, bb_inds, bb_data};
  if (threads < 1) threads = 1;
  auto work = [&](int t) {
    const int64_t lo = first + count * t / threads, hi = first + count * (t + 1) / threads;
    const int K = num_dates * num_und;
    std::vector<float> gauss(K), bbrow(num_dates), bb(K), prices(K);
    std::vector<double> acc(num_models);
    for (int64_t it = lo; it < hi; it++) {
      for (int m = 0; m < num_models; m++) acc[m] = 0.0;
      op_path(q, (int32_t)(it + 1), gauss.data(), bbrow.data(), bb.data(), prices.data(), acc.data());
      for (int m = 0; m < num_models; m++) out[(it - first) * num_models + m] = (float)acc[m];
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < threads; t++) pool.emplace_back(work, t);
  work(0);
  for (auto& th : pool) th.join();
}

// One path's payoff per model (f32, before the mean) -- for per-path checks.
void lvc_oracle_op_path(int contract, int num_bits, int num_models, int num_und, int num_dates, int num_discts,
                        const int32_t* dir_vs, const float* md_cs, const float* md_vols, const float* md_drifts,
                        const float* md_sts, const float* md_detvals, const float* md_discts, const int32_t* bb_inds,
                        const float* bb_data, int32_t n, double* payoffs) {
  OpArgs q{contract, 0, num_bits, num_models, num_und, num_dates, num_discts, dir_vs, md_cs, md_vols, md_drifts,
           md_sts, md_detvals, md_discts, bb_inds, bb_data};
  const int K = num_dates * num_und;
  std::vector<float> gauss(K), bbrow(num_dates), bb(K), prices(K);
  for (int m = 0; m < num_models; m++) payoffs[m] = 0.0;
  op_path(q, n, gauss.data(), bbrow.data(), bb.data(), prices.data(), payoffs);
}

}  // extern "C"
