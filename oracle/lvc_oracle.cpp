// LocVolCalib CPU oracle -- TEST INFRASTRUCTURE ONLY.
//
// A line-by-line restatement of the reference program finpar/LocVolCalib.fut
// (diku-dk/futhark-benchmarks), templated on the element type so that the same
// source gives the reference's own f32 arithmetic and an f64 twin.  It is the
// checker for the CUDA engine (tests, the smoke check) and the timed CPU
// baseline of bench.py; no product code path links or calls it.
//
// Fidelity rules followed here:
//   * every array the reference materialises is materialised (MuX, VarX, MuY,
//     VarY, the transposes), and every formula keeps the reference's operand
//     order and association (build with -ffp-contract=off so no FMA is formed);
//   * tridagPar is evaluated as the three scans of LocVolCalib.fut:68-124,
//     each scan folded left to right with the reference's operator and neutral
//     element (a sequential evaluation of the same scan);
//   * tridagSeq (misc/ocean-sim/tridiag.fut:81-95) is provided as the second,
//     independent formulation used to cross-check the scan form.
//
// Exported C ABI (all functions are re-entrant; the multi-strike entries spread
// independent strikes over `threads` host threads with a dynamic schedule,
// threads <= 0 meaning every hardware thread):
//   lvc_oracle_main_f32 / _f64           : the reference `main` (:238-252)
//   lvc_oracle_value_f32 / _f64          : the reference `value` (:211-236)
//   lvc_oracle_batch_f64                 : many calibrations, prices concatenated
//   lvc_oracle_tridag_{par,par4,seq}_{f32,f64}: row-batched tridiagonal solvers
//     (par: LocVolCalib.fut's tridagPar; par4: misc/ocean-sim/tridiag.fut's)
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <atomic>
#include <thread>

namespace {

inline float f_log(float x) { return logf(x); }
inline double f_log(double x) { return log(x); }
inline float f_exp(float x) { return expf(x); }
inline double f_exp(double x) { return exp(x); }
inline float f_sqrt(float x) { return sqrtf(x); }
inline double f_sqrt(double x) { return sqrt(x); }
inline float f_max(float a, float b) { return fmaxf(a, b); }
inline double f_max(double a, double b) { return fmax(a, b); }

// Futhark's i32.f32 / i32.f64: truncation toward zero.  Values outside the
// i32 range (or NaN) are clamped so the oracle never invokes C undefined
// behaviour; the engine rejects such inputs before any work is done.
template <typename T> int32_t to_i32(T v) {
  if (!(v == v)) return 0;
  if (v >= (T)2147483647.0) return 2147483647;
  if (v <= (T)-2147483648.0) return (int32_t)(-2147483647 - 1);
  return (int32_t)v;
}

// Dynamic-schedule parallel loop over [0, n) on `threads` std::threads.
template <typename F> void parallel_for(int64_t n, int threads, F&& body) {
  if (threads <= 0) threads = (int)std::thread::hardware_concurrency();
  if (threads <= 1 || n <= 1) {
    for (int64_t k = 0; k < n; k++) body(k);
    return;
  }
  if ((int64_t)threads > n) threads = (int)n;
  std::atomic<int64_t> next{0};
  std::vector<std::thread> pool;
  pool.reserve(threads);
  for (int w = 0; w < threads; w++)
    pool.emplace_back([&]() {
      for (int64_t k = next.fetch_add(1); k < n; k = next.fetch_add(1)) body(k);
    });
  for (auto& th : pool) th.join();
}

template <typename T> struct Grid {
  int32_t xindex = 0, yindex = 0;
  std::vector<T> x, y, timeline;
};

// finpar/LocVolCalib.fut:12-23 (initGrid)
template <typename T>
Grid<T> init_grid(T s0, T alpha, T nu, T t, int64_t numX, int64_t numY, int64_t numT) {
  Grid<T> g;
  const T logAlpha = f_log(alpha);
  g.timeline.resize(numT);
  for (int64_t i = 0; i < numT; i++)
    g.timeline[i] = t * (T)i / ((T)numT - (T)1.0);
  const T stdX = (T)20.0 * alpha * s0 * f_sqrt(t);
  const T stdY = (T)10.0 * nu * f_sqrt(t);
  const T dx = stdX / (T)numX;
  const T dy = stdY / (T)numY;
  g.xindex = to_i32<T>(s0 / dx);
  g.yindex = (int32_t)numY / 2;
  g.x.resize(numX);
  g.y.resize(numY);
  for (int64_t i = 0; i < numX; i++)
    g.x[i] = (T)i * dx - (T)g.xindex * dx + s0;
  for (int64_t i = 0; i < numY; i++)
    g.y[i] = (T)i * dy - (T)g.yindex * dy + logAlpha;
  return g;
}

// finpar/LocVolCalib.fut:26-44 (initOperator); D and DD are [n][3] row-major.
template <typename T>
void init_operator(const std::vector<T>& x, std::vector<T>& D, std::vector<T>& DD) {
  const int64_t n = (int64_t)x.size();
  D.assign(n * 3, (T)0);
  DD.assign(n * 3, (T)0);
  {
    const T dxu = x[1] - x[0];
    D[0] = (T)0.0;
    D[1] = (T)-1.0 / dxu;
    D[2] = (T)1.0 / dxu;
  }
  for (int64_t i = 1; i <= n - 2; i++) {
    const T dxl = x[i] - x[i - 1];
    const T dxu = x[i + 1] - x[i];
    D[i * 3 + 0] = -dxu / dxl / (dxl + dxu);
    D[i * 3 + 1] = (dxu / dxl - dxl / dxu) / (dxl + dxu);
    D[i * 3 + 2] = dxl / dxu / (dxl + dxu);
    DD[i * 3 + 0] = (T)2.0 / dxl / (dxl + dxu);
    DD[i * 3 + 1] = (T)-2.0 * ((T)1.0 / dxl + (T)1.0 / dxu) / (dxl + dxu);
    DD[i * 3 + 2] = (T)2.0 / dxu / (dxl + dxu);
  }
  {
    const T dxl = x[n - 1] - x[n - 2];
    D[(n - 1) * 3 + 0] = (T)-1.0 / dxl;
    D[(n - 1) * 3 + 1] = (T)1.0 / dxl;
    D[(n - 1) * 3 + 2] = (T)0.0;
  }
}

// finpar/LocVolCalib.fut:68-124 (tridagPar), the three scans folded left to
// right.  `out` may alias `y`.  `bp`/`yp` are caller scratch of length n.
template <typename T>
void tridag_par(int64_t n, const T* a, const T* b, const T* c, const T* y, T* out,
                T* bp, T* yp) {
  // Recurrence 1: 2x2 (normalised Moebius) matrix scan, :74-91.
  const T b0 = b[0];
  T s1 = (T)0.0, s2 = (T)0.0, s3 = (T)1.0;  // neutral element (0,0,1)
  for (int64_t i = 0; i < n; i++) {
    T m1, m2, m3;
    if (0 < i) {
      const T bi = (T)1 / b[i];
      m1 = -a[i] * c[i - 1] * bi;
      m2 = bi;
      m3 = (T)0.0;
    } else {
      m1 = (T)0.0;
      m2 = (T)0.0;
      m3 = (T)1.0;
    }
    const T value = (T)1.0 / ((T)1.0 + m1 * s2);
    const T n1 = (s1 + m1 * s3) * value;
    const T n2 = (m2 + m3 * s2) * value;
    const T n3 = (m2 * s1 + m3 * s3) * value;
    s1 = n1;
    s2 = n2;
    s3 = n3;
    bp[i] = (b0 + s1) / (s2 * b0 + s3);
  }
  // Recurrence 2: forward linear-function-composition scan, :96-106.
  const T y0 = y[0];
  T c0 = (T)0.0, c1 = (T)1.0;  // neutral element (0,1)
  for (int64_t i = 0; i < n; i++) {
    T l0, l1;
    if (0 < i) {
      l0 = y[i];
      l1 = (T)0.0 - a[i] / bp[i - 1];
    } else {
      l0 = (T)0.0;
      l1 = (T)1.0;
    }
    const T n0 = l0 + l1 * c0;
    const T n1 = c1 * l1;
    c0 = n0;
    c1 = n1;
    yp[i] = c0 + c1 * y0;
  }
  // Recurrence 3: backward scan over the reversed index, :111-123.
  const T yn = yp[n - 1] / bp[n - 1];
  c0 = (T)0.0;
  c1 = (T)1.0;
  for (int64_t k = 0; k < n; k++) {
    const int64_t i = n - k - 1;
    T l0, l1;
    if (0 < k) {
      l0 = yp[i] / bp[i];
      l1 = (T)0.0 - c[i] / bp[i];
    } else {
      l0 = (T)0.0;
      l1 = (T)1.0;
    }
    const T n0 = l0 + l1 * c0;
    const T n1 = c1 * l1;
    c0 = n0;
    c1 = n1;
    out[i] = c0 + c1 * yn;  // the reverse of :122-123
  }
}

// misc/ocean-sim/tridiag.fut:4-79 (the tridagPar of the tridiagonal test
// program): recurrence 1 as a scan of 4-tuple matrices normalised by
// 1/(a0*b0) (:9-33), recurrences 2 and 3 as in tridag_par above (:38-79); the
// scans folded left to right, accumulator as the operator's first argument.
template <typename T>
void tridag_par4(int64_t n, const T* a, const T* b, const T* c, const T* y, T* out,
                 T* bp, T* yp) {
  const T b0 = b[0];
  T s0 = (T)1.0, s1 = (T)0.0, s2 = (T)0.0, s3 = (T)1.0;  // neutral element (1,0,0,1)
  for (int64_t i = 0; i < n; i++) {
    T m0, m1, m2, m3;
    if (0 < i) {
      m0 = b[i];
      m1 = (T)0.0 - a[i] * c[i - 1];
      m2 = (T)1.0;
      m3 = (T)0.0;
    } else {
      m0 = (T)1.0;
      m1 = (T)0.0;
      m2 = (T)0.0;
      m3 = (T)1.0;
    }
    const T value = (T)1.0 / (s0 * m0);
    const T n0 = (m0 * s0 + m1 * s2) * value;
    const T n1 = (m0 * s1 + m1 * s3) * value;
    const T n2 = (m2 * s0 + m3 * s2) * value;
    const T n3 = (m2 * s1 + m3 * s3) * value;
    s0 = n0;
    s1 = n1;
    s2 = n2;
    s3 = n3;
    bp[i] = (s0 * b0 + s1) / (s2 * b0 + s3);
  }
  const T y0 = y[0];
  T c0 = (T)0.0, c1 = (T)1.0;
  for (int64_t i = 0; i < n; i++) {
    T l0, l1;
    if (0 < i) {
      l0 = y[i];
      l1 = (T)0.0 - a[i] / bp[i - 1];
    } else {
      l0 = (T)0.0;
      l1 = (T)1.0;
    }
    const T n0 = l0 + l1 * c0;
    const T n1 = c1 * l1;
    c0 = n0;
    c1 = n1;
    yp[i] = c0 + c1 * y0;
  }
  const T yn = yp[n - 1] / bp[n - 1];
  c0 = (T)0.0;
  c1 = (T)1.0;
  for (int64_t k = 0; k < n; k++) {
    const int64_t i = n - k - 1;
    T l0, l1;
    if (0 < k) {
      l0 = yp[i] / bp[i];
      l1 = (T)0.0 - c[i] / bp[i];
    } else {
      l0 = (T)0.0;
      l1 = (T)1.0;
    }
    const T n0 = l0 + l1 * c0;
    const T n1 = c1 * l1;
    c0 = n0;
    c1 = n1;
    out[i] = c0 + c1 * yn;
  }
}

// misc/ocean-sim/tridiag.fut:81-95 (tridagSeq): normalised Thomas algorithm.
template <typename T>
void tridag_seq(int64_t m, const T* a, const T* b, const T* c, const T* y, T* out,
                T* cp, T* yp) {
  cp[0] = c[0] / b[0];
  yp[0] = y[0] / b[0];
  for (int64_t i = 1; i < m; i++) {
    const T norm_factor = (T)1.0 / (b[i] - a[i] * cp[i - 1]);
    cp[i] = c[i] * norm_factor;
    yp[i] = (y[i] - a[i] * yp[i - 1]) * norm_factor;
  }
  out[m - 1] = yp[m - 1];
  for (int64_t i = m - 2; i >= 0; i--) out[i] = yp[i] - cp[i] * out[i + 1];
}

// ---------------------------------------------------------------------------
// misc/ocean-sim/tke.fut:64-348 (entry main, DTYPE = f32 via typeinst32): the
// turbulent-kinetic-energy step of the ocean model.  Arrays are row-major
// [xdim][ydim][zdim] (z innermost), [xdim][ydim] and [n].  Every expression
// keeps the reference's operand order (no contraction); the vertical
// tridiagonal solve is tridag_par4 (misc/ocean-sim/tridiag.fut:4-79) over
// the z columns, as tke.fut:4-17 maps tridagPar over them.
// ---------------------------------------------------------------------------
template <typename T>
static T tke_limiter(T cr) {  // tke.fut:19-20
  return std::max((T)0, std::max(std::min((T)1, (T)2 * cr), std::min((T)2, cr)));
}

template <typename T>
static T tke_calcflux(T velfac, T velS, T dt_tracer, T dx, T varS, T varSM1, T varSP1, T varSP2, T maskS,
                      T maskSM1, T maskSP1) {  // tke.fut:22-41
  const T scaledVel = velfac * velS;
  const T uCFL = std::fabs(scaledVel * dt_tracer / dx);
  const T rjp = (varSP2 - varSP1) * maskSP1;
  const T rj = (varSP1 - varS) * maskS;
  const T rjm = (varS - varSM1) * maskSM1;
  const T epsilon = (T)0.00000000000000000001;
  const T divisor = (std::fabs(rj) < epsilon) ? epsilon : rj;
  T cr = (velS > 0) ? rjm / divisor : rjp / divisor;
  cr = tke_limiter<T>(cr);
  return scaledVel * (varSP1 + varS) * (T)0.5 - std::fabs(scaledVel) * (((T)1.0 - cr) + uCFL * cr) * rj * (T)0.5;
}

template <typename T>
static void tke_main(int X, int Y, int Z, const T* tketau, const T* tketaup1_in, const T* dtketau_in,
                     const T* dtketaum1, const T* utau, const T* vtau, const T* wtau, const T* maskU,
                     const T* maskV, const T* maskW, const T* dxt, const T* dxu, const T* dyt, const T* dyu,
                     const T* dzt, const T* dzw, const T* cost, const T* cosu, const int32_t* kbot,
                     const T* kappaM, const T* mxl, const T* forc, const T* forc_tke_surface, T* tketaup1,
                     T* dtketau, T* tke_surf_corr) {
  const T dt_tracer = 1, dt_mom = 1, AB_eps = (T)0.1, alpha_tke = 1, c_eps = (T)0.7, K_h_tke = 2000;
  const T dt_tke = dt_mom;
  const int64_t N = (int64_t)X * Y * Z;
  auto I3 = [&](int x, int y, int z) { return ((int64_t)x * Y + y) * Z + z; };
  auto I2 = [&](int x, int y) { return (int64_t)x * Y + y; };
  auto interior = [&](int x, int y) { return x >= 2 && x < X - 2 && y >= 2 && y < Y - 2; };
  std::vector<T> delta(N), a(N), b(N), c(N), d(N), sol(N), fe(N), fn(N), ft(N);
  for (int x = 0; x < X; x++)  // :103-108
    for (int y = 0; y < Y; y++)
      for (int z = 0; z < Z; z++)
        delta[I3(x, y, z)] = (interior(x, y) && z < Z - 1)
                                 ? dt_tke / dzt[z + 1] * alpha_tke * (T)0.5 *
                                       (kappaM[I3(x, y, z)] + kappaM[I3(x, y, z + 1)])
                                 : (T)0;
  for (int x = 0; x < X; x++)
    for (int y = 0; y < Y; y++)
      for (int z = 0; z < Z; z++) {
        const int64_t i = I3(x, y, z);
        const T sqrttke = std::sqrt(std::max((T)0, tketau[i]));
        T av = 0, bv = 0, cv = 0, dv = 0;
        if (interior(x, y)) {
          const int ks = kbot[I2(x, y)] - 1;
          const bool land = ks >= 0;
          const bool edge = land && z == ks;
          const bool water = land && z >= ks;
          // a_tri (:109-122)
          if (edge || !water) av = 0;
          else if (z > 0 && z < Z - 1) av = -delta[I3(x, y, z - 1)] / dzw[z];
          else if (z == Z - 1) av = -delta[I3(x, y, z - 1)] / ((T)0.5 * dzw[z]);
          else av = 0;
          // b_tri (:123-146)
          if (!water) bv = 1;
          else if (edge) bv = (T)1 + delta[i] / dzw[z] + dt_tke * c_eps / mxl[i] * sqrttke;
          else if (z > 0 && z < Z - 1)
            bv = (T)1 + (delta[i] + delta[I3(x, y, z - 1)]) / dzw[z] + dt_tke * c_eps * sqrttke / mxl[i];
          else if (z == Z - 1)
            bv = (T)1 + delta[I3(x, y, z - 1)] / ((T)0.5 * dzw[z]) + dt_tke * c_eps / mxl[i] * sqrttke;
          else bv = 0;
          // c_tri (:187-196)
          if (z < Z - 1) cv = water ? -delta[i] / dzw[z] : (T)0;
          // d_tri (:197-210)
          if (water) {
            const T tmp = tketau[i] + dt_tke * forc[i];
            dv = (z == Z - 1) ? tmp + dt_tke * forc_tke_surface[I2(x, y)] / ((T)0.5 * dzw[z]) : tmp;
          }
        }
        a[i] = av;
        b[i] = bv;
        c[i] = cv;
        d[i] = dv;
      }
  {  // sol = tridiag a b c d (:211), tridagPar along z
    std::vector<T> s1(Z), s2(Z);
    for (int64_t col = 0; col < (int64_t)X * Y; col++)
      tridag_par4<T>(Z, &a[col * Z], &b[col * Z], &c[col * Z], &d[col * Z], &sol[col * Z], s1.data(), s2.data());
  }
  for (int x = 0; x < X; x++)  // :212-218
    for (int y = 0; y < Y; y++)
      for (int z = 0; z < Z; z++) {
        const int64_t i = I3(x, y, z);
        const int ks = kbot[I2(x, y)] - 1;
        const bool water = ks >= 0 && z >= ks;
        tketaup1[i] = (interior(x, y) && water) ? sol[i] : tketaup1_in[i];
      }
  for (int x = 0; x < X; x++)  // :219-226
    for (int y = 0; y < Y; y++) {
      T v = 0;
      if (interior(x, y)) {
        const T tke_val = tketaup1[I3(x, y, Z - 1)];
        v = tke_val < 0 ? -tke_val * (T)0.5 * dzw[Z - 1] / dt_tke : (T)0;
      }
      tke_surf_corr[I2(x, y)] = v;
    }
  for (int x = 0; x < X; x++)  // :227-235
    for (int y = 0; y < Y; y++)
      if (interior(x, y)) {
        T& v = tketaup1[I3(x, y, Z - 1)];
        v = v < 0 ? (T)0 : v;
      }
  for (int x = 0; x < X; x++)  // lateral diffusion fluxes :236-251
    for (int y = 0; y < Y; y++)
      for (int z = 0; z < Z; z++) {
        const int64_t i = I3(x, y, z);
        fe[i] = (x < X - 1) ? K_h_tke * (tketau[I3(x + 1, y, z)] - tketau[i]) / (cost[y] * dxu[x]) * maskU[i] : (T)0;
        fn[i] = (y < Y - 1) ? K_h_tke * (tketau[I3(x, y + 1, z)] - tketau[i]) / dyu[y] * maskV[i] * cosu[y] : (T)0;
      }
  for (int x = 0; x < X; x++)  // :252-263
    for (int y = 0; y < Y; y++) {
      if (!interior(x, y)) continue;
      const int z = Z - 1;
      const int64_t i = I3(x, y, z);
      tketaup1[i] = tketaup1[i] + dt_tke * maskW[i] *
                                      ((fe[i] - fe[I3(x - 1, y, z)]) / (cost[y] * dxt[x]) +
                                       (fn[i] - fn[I3(x, y - 1, z)]) / (cost[y] * dyt[y]));
    }
  for (int x = 0; x < X; x++)  // advection fluxes :264-319
    for (int y = 0; y < Y; y++)
      for (int z = 0; z < Z; z++) {
        const int64_t i = I3(x, y, z);
        T e = 0, n = 0, t = 0;
        if (x >= 1 && x < X - 2 && y >= 2 && y < Y - 2) {
          const T dx = cost[y] * dxt[x];
          const T mWm1 = maskW[I3(x - 1, y, z)], mWs = maskW[i], mWp1 = maskW[I3(x + 1, y, z)],
                  mWp2 = maskW[I3(x + 2, y, z)];
          const T mtr = x < X - 1 ? mWs * mWp1 : (T)0;
          const T mtrP1 = x < X - 1 ? mWp1 * mWp2 : (T)0;
          const T mtrM1 = x < X - 1 ? mWm1 * mWs : (T)0;
          e = tke_calcflux<T>((T)1, utau[i], dt_tracer, dx, tketau[i], tketau[I3(x - 1, y, z)],
                              tketau[I3(x + 1, y, z)], tketau[I3(x + 2, y, z)], mtr, mtrM1, mtrP1);
        }
        if (y >= 1 && y < Y - 2 && x >= 2 && x < X - 2) {
          const T dx = cost[y] * dyt[y];
          const T mWm1 = maskW[I3(x, y - 1, z)], mWs = maskW[i], mWp1 = maskW[I3(x, y + 1, z)],
                  mWp2 = maskW[I3(x, y + 2, z)];
          const T mtr = y < Y - 1 ? mWs * mWp1 : (T)0;
          const T mtrP1 = y < Y - 1 ? mWp1 * mWp2 : (T)0;
          const T mtrM1 = y < Y - 1 ? mWm1 * mWs : (T)0;
          n = tke_calcflux<T>(cosu[y], vtau[i], dt_tracer, dx, tketau[i], tketau[I3(x, y - 1, z)],
                              tketau[I3(x, y + 1, z)], tketau[I3(x, y + 2, z)], mtr, mtrM1, mtrP1);
        }
        if (z < Z - 1 && interior(x, y)) {
          const T varSM1 = z != 0 ? tketau[I3(x, y, z - 1)] : (T)0;
          const T varS = tketau[i];
          const T varSP2 = z < Z - 2 ? tketau[I3(x, y, z + 2)] : (T)0;
          const T varSP1 = tketau[I3(x, y, z + 1)];
          const T mWm1 = z != 0 ? maskW[I3(x, y, z - 1)] : (T)0;
          const T mWs = maskW[i];
          const T mWp1 = maskW[I3(x, y, z + 1)];
          const T mWp2 = z < Z - 2 ? maskW[I3(x, y, z + 2)] : (T)0;
          t = tke_calcflux<T>((T)1, wtau[i], dt_tracer, dzw[z], varS, varSM1, varSP1, varSP2, mWs * mWp1,
                              mWm1 * mWs, mWp1 * mWp2);
        }
        fe[i] = e;
        fn[i] = n;
        ft[i] = t;
      }
  for (int x = 0; x < X; x++)  // dtketau :320-340
    for (int y = 0; y < Y; y++)
      for (int z = 0; z < Z; z++) {
        const int64_t i = I3(x, y, z);
        const T tmp = interior(x, y)
                          ? maskW[i] * (-(fe[i] - fe[I3(x - 1, y, z)]) / (cost[y] * dxt[x]) -
                                        (fn[i] - fn[I3(x, y - 1, z)]) / (cost[y] * dyt[y]))
                          : dtketau_in[i];
        const T z0 = z == 0 ? tmp - ft[I3(x, y, 0)] / dzw[0] : tmp;
        const T zm = (z >= 1 && z < Z - 1) ? z0 - (ft[i] - ft[I3(x, y, z - 1)]) / dzw[z] : z0;
        dtketau[i] = (z == Z - 1) ? zm - (ft[i] - ft[I3(x, y, z - 1)]) / ((T)0.5 * dzw[z]) : zm;
      }
  for (int64_t i = 0; i < N; i++)  // :341-347
    tketaup1[i] = tketaup1[i] + dt_tracer * (((T)1.5 + AB_eps) * dtketau[i] - ((T)0.5 + AB_eps) * dtketaum1[i]);
}

// finpar/LocVolCalib.fut:126-153 (explicitMethod).  Arrays are row-major
// [rows][m]; D/DD are [m][3].
template <typename T>
void explicit_method(int64_t rows, int64_t m, const T* D, const T* DD, const T* mu,
                     const T* var, const T* result, T* out) {
  for (int64_t r = 0; r < rows; r++) {
    const T* mu_row = mu + r * m;
    const T* var_row = var + r * m;
    const T* res_row = result + r * m;
    T* out_row = out + r * m;
    for (int64_t j = 0; j < m; j++) {
      const T* dx = D + j * 3;
      const T* dxx = DD + j * 3;
      const T mu_ = mu_row[j], var_ = var_row[j];
      const T c1 = (0 < j) ? (mu_ * dx[0] + (T)0.5 * var_ * dxx[0]) * res_row[j - 1] : (T)0.0;
      const T c3 = (j < (m - 1)) ? (mu_ * dx[2] + (T)0.5 * var_ * dxx[2]) * res_row[j + 1]
                                 : (T)0.0;
      const T c2 = (mu_ * dx[1] + (T)0.5 * var_ * dxx[1]) * res_row[j];
      out_row[j] = c1 + c2 + c3;
    }
  }
}

// finpar/LocVolCalib.fut:156-178 (implicitMethod), in place on u [rows][m].
template <typename T>
void implicit_method(int64_t rows, int64_t m, const T* D, const T* DD, const T* mu,
                     const T* var, T* u, T dtInv, bool use_seq) {
  std::vector<T> a(m), b(m), c(m), s1(m), s2(m);
  for (int64_t r = 0; r < rows; r++) {
    const T* mu_row = mu + r * m;
    const T* var_row = var + r * m;
    for (int64_t j = 0; j < m; j++) {
      const T* d = D + j * 3;
      const T* dd = DD + j * 3;
      const T mu_ = mu_row[j], var_ = var_row[j];
      a[j] = (T)0.0 - (T)0.5 * (mu_ * d[0] + (T)0.5 * var_ * dd[0]);
      b[j] = dtInv - (T)0.5 * (mu_ * d[1] + (T)0.5 * var_ * dd[1]);
      c[j] = (T)0.0 - (T)0.5 * (mu_ * d[2] + (T)0.5 * var_ * dd[2]);
    }
    T* row = u + r * m;
    if (use_seq)
      tridag_seq<T>(m, a.data(), b.data(), c.data(), row, row, s1.data(), s2.data());
    else
      tridag_par<T>(m, a.data(), b.data(), c.data(), row, row, s1.data(), s2.data());
  }
}

template <typename T>
void transpose(int64_t rows, int64_t cols, const T* in, T* out) {
  for (int64_t r = 0; r < rows; r++)
    for (int64_t c = 0; c < cols; c++) out[c * rows + r] = in[r * cols + c];
}

// finpar/LocVolCalib.fut:211-236 (value), with updateParams (:50-66) and
// rollback (:180-209) inlined in the time loop.
template <typename T>
T value(int64_t numX, int64_t numY, int64_t numT, T s0, T strike, T t, T alpha, T nu,
        T beta, bool use_seq) {
  const Grid<T> g = init_grid<T>(s0, alpha, nu, t, numX, numY, numT);
  std::vector<T> Dx, Dxx, Dy, Dyy;
  init_operator<T>(g.x, Dx, Dxx);
  init_operator<T>(g.y, Dy, Dyy);
  const int64_t XY = numX * numY;
  // setPayoff, :46-47: [numY][numX]
  std::vector<T> res(XY);
  for (int64_t j = 0; j < numY; j++)
    for (int64_t i = 0; i < numX; i++) res[j * numX + i] = f_max(g.x[i] - strike, (T)0.0);

  std::vector<T> muX(XY), varX(XY), muY(XY), varY(XY);
  std::vector<T> u(XY), v(XY), resT(XY), y(XY), tmp(XY);
  for (int64_t k = numT - 2; k >= 0; k--) {  // reverse (zip (init tl) (tail tl))
    const T tnow = g.timeline[k], tnext = g.timeline[k + 1];
    // updateParams, :50-66
    for (int64_t i = 0; i < XY; i++) {
      muY[i] = (T)0.0;
      varY[i] = nu * nu;
      muX[i] = (T)0.0;
    }
    for (int64_t j = 0; j < numY; j++) {
      const T yj = g.y[j];
      for (int64_t i = 0; i < numX; i++)
        varX[j * numX + i] =
            f_exp((T)2.0 * (beta * f_log(g.x[i]) + yj - (T)0.5 * nu * nu * tnow));
    }
    // rollback, :180-209
    const T dtInv = (T)1.0 / (tnext - tnow);
    explicit_method<T>(numY, numX, Dx.data(), Dxx.data(), muX.data(), varX.data(), res.data(),
                       u.data());
    for (int64_t i = 0; i < XY; i++) u[i] = dtInv * res[i] + (T)0.5 * u[i];
    transpose<T>(numY, numX, res.data(), resT.data());
    explicit_method<T>(numX, numY, Dy.data(), Dyy.data(), muY.data(), varY.data(), resT.data(),
                       v.data());  // v is [numX][numY]
    transpose<T>(numX, numY, v.data(), tmp.data());  // transpose v -> [numY][numX]
    for (int64_t i = 0; i < XY; i++) u[i] = u[i] + tmp[i];
    implicit_method<T>(numY, numX, Dx.data(), Dxx.data(), muX.data(), varX.data(), u.data(),
                       dtInv, use_seq);
    transpose<T>(numY, numX, u.data(), tmp.data());  // transpose u -> [numX][numY]
    for (int64_t i = 0; i < XY; i++) y[i] = dtInv * tmp[i] - (T)0.5 * v[i];
    implicit_method<T>(numX, numY, Dy.data(), Dyy.data(), muY.data(), varY.data(), y.data(),
                       dtInv, use_seq);
    transpose<T>(numX, numY, y.data(), res.data());
  }
  return res[(int64_t)g.yindex * numX + g.xindex];
}

// finpar/LocVolCalib.fut:238-252 (main); strikes are 0.001 * i in type T.
template <typename T>
void main_entry(int32_t outer, int32_t numX, int32_t numY, int32_t numT, T s0, T t, T alpha,
                T nu, T beta, T* out, int threads, bool use_seq) {
  parallel_for(outer, threads, [&](int64_t i) {
    const T strike = (T)0.001 * (T)i;
    out[i] = value<T>(numX, numY, numT, s0, strike, t, alpha, nu, beta, use_seq);
  });
}

// Returns 0 on success, 1 if the grid indices the reference reads
// (res[myYindex, myXindex], :236) or the operator stencils (:27,39) would be
// out of bounds -- the cases where the reference program fails.
int check_sizes(int32_t outer, int32_t numX, int32_t numY, int32_t numT) {
  if (outer < 0 || numX < 3 || numY < 3 || numT < 1) return 1;
  return 0;
}

template <typename T>
int main_checked(int32_t outer, int32_t numX, int32_t numY, int32_t numT, T s0, T t,
                        T alpha, T nu, T beta, T* out, int threads, int use_seq) {
  if (check_sizes(outer, numX, numY, numT)) return 1;
  const Grid<T> g = init_grid<T>(s0, alpha, nu, t, numX, 3, 2);
  if (g.xindex < 0 || g.xindex >= numX) return 1;
  main_entry<T>(outer, numX, numY, numT, s0, t, alpha, nu, beta, out, threads, use_seq != 0);
  return 0;
}

}  // namespace

extern "C" {

int lvc_oracle_main_f32(int32_t outer, int32_t numX, int32_t numY, int32_t numT, float s0,
                        float t, float alpha, float nu, float beta, float* out, int threads,
                        int use_seq) {
  return main_checked<float>(outer, numX, numY, numT, s0, t, alpha, nu, beta, out, threads,
                             use_seq);
}

int lvc_oracle_main_f64(int32_t outer, int32_t numX, int32_t numY, int32_t numT, double s0,
                        double t, double alpha, double nu, double beta, double* out,
                        int threads, int use_seq) {
  return main_checked<double>(outer, numX, numY, numT, s0, t, alpha, nu, beta, out, threads,
                              use_seq);
}

double lvc_oracle_value_f64(int32_t numX, int32_t numY, int32_t numT, double s0, double strike,
                            double t, double alpha, double nu, double beta, int use_seq) {
  return value<double>(numX, numY, numT, s0, strike, t, alpha, nu, beta, use_seq != 0);
}

float lvc_oracle_value_f32(int32_t numX, int32_t numY, int32_t numT, float s0, float strike,
                           float t, float alpha, float nu, float beta, int use_seq) {
  return value<float>(numX, numY, numT, s0, strike, t, alpha, nu, beta, use_seq != 0);
}

// The grid index the reference reads its price from (:20), for tests.
int lvc_oracle_xindex_f64(int32_t numX, double s0, double t, double alpha) {
  return init_grid<double>(s0, alpha, 0.5, t, numX, 3, 2).xindex;
}

// Many calibrations: instance list of (calibration, strike index) pairs is
// flattened in calibration order; prices are written at offsets[c] + i.
// Work items are independent strikes (OpenMP dynamic schedule).
int lvc_oracle_batch_f64(int32_t n_calib, const int32_t* outer, const int32_t* numX,
                         const int32_t* numY, const int32_t* numT, const double* s0,
                         const double* t, const double* alpha, const double* nu,
                         const double* beta, const int64_t* offsets, double* out, int threads) {
  int64_t total = 0;
  for (int32_t c = 0; c < n_calib; c++) {
    if (check_sizes(outer[c], numX[c], numY[c], numT[c])) return 1;
    total += outer[c];
  }
  std::vector<int32_t> item_c(total), item_i(total);
  {
    int64_t k = 0;
    for (int32_t c = 0; c < n_calib; c++)
      for (int32_t i = 0; i < outer[c]; i++) {
        item_c[k] = c;
        item_i[k] = i;
        k++;
      }
  }
  parallel_for(total, threads, [&](int64_t k) {
    const int32_t c = item_c[k], i = item_i[k];
    const double strike = 0.001 * (double)(int64_t)i;
    out[offsets[c] + i] = value<double>(numX[c], numY[c], numT[c], s0[c], strike, t[c],
                                        alpha[c], nu[c], beta[c], false);
  });
  return 0;
}

// Row-batched solvers over [rows][n] arrays (the tridagNested* entry points of
// misc/ocean-sim/tridiag-test.fut:14-26).
#define LVC_TRIDAG_BATCH(NAME, T, FN)                                                    \
  void NAME(int64_t rows, int64_t n, const T* a, const T* b, const T* c, const T* y,     \
            T* out) {                                                                    \
    std::vector<T> s1(n), s2(n);                                                         \
    for (int64_t r = 0; r < rows; r++)                                                   \
      FN<T>(n, a + r * n, b + r * n, c + r * n, y + r * n, out + r * n, s1.data(),       \
            s2.data());                                                                  \
  }
LVC_TRIDAG_BATCH(lvc_oracle_tridag_par_f32, float, tridag_par)
LVC_TRIDAG_BATCH(lvc_oracle_tridag_par_f64, double, tridag_par)
LVC_TRIDAG_BATCH(lvc_oracle_tridag_seq_f32, float, tridag_seq)
LVC_TRIDAG_BATCH(lvc_oracle_tridag_seq_f64, double, tridag_seq)
LVC_TRIDAG_BATCH(lvc_oracle_tridag_par4_f32, float, tridag_par4)
LVC_TRIDAG_BATCH(lvc_oracle_tridag_par4_f64, double, tridag_par4)

// tke.fut's entry main (f32): the three arrays it computes; the other four
// outputs are its inputs tketau, tketaum1, dtketaup1, dtketaum1 unchanged.
void lvc_oracle_tke_f32(int X, int Y, int Z, const float* tketau, const float* tketaup1_in,
                        const float* dtketau_in, const float* dtketaum1, const float* utau, const float* vtau,
                        const float* wtau, const float* maskU, const float* maskV, const float* maskW,
                        const float* dxt, const float* dxu, const float* dyt, const float* dyu, const float* dzt,
                        const float* dzw, const float* cost, const float* cosu, const int32_t* kbot,
                        const float* kappaM, const float* mxl, const float* forc, const float* forc_tke_surface,
                        float* tketaup1, float* dtketau, float* tke_surf_corr) {
  tke_main<float>(X, Y, Z, tketau, tketaup1_in, dtketau_in, dtketaum1, utau, vtau, wtau, maskU, maskV, maskW, dxt,
                  dxu, dyt, dyu, dzt, dzw, cost, cosu, kbot, kappaM, mxl, forc, forc_tke_surface, tketaup1,
                  dtketau, tke_surf_corr);
}

int lvc_oracle_max_threads(void) { return (int)std::thread::hardware_concurrency(); }

}  // extern "C"
