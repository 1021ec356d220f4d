// Quasiparticle equation on the GPU: analytic continuation of the diagonal self-energy from
// the imaginary to the real frequency axis by an N-point Pade approximant (Thiele's
// reciprocal differences, J. Low Temp. Phys. 29, 179 (1977)), and the solution of
//     E = V_hf + Re Sigma(E - mu + i eta)
// per (spin, k, band) element, one thread per element.
//
// Reference: analyt_cont::pade_t (src/numerics/ac/pade/pade_t.hpp: fit :133-170, evaluate
// :100-120), solved for by solve_qp_eqn (src/methods/SCF/qp_scf_common.cpp:150-311) with
// qp_eqn_bisection (:678-748, "sc"), qp_eqn_secant (:629-676, "sc_newton"),
// qp_eqn_linearized (:619-627) and qp_eqn_spectral (:560-617).  The reference carries the
// continued fraction in 100-digit decimal arithmetic; here it runs in double-double
// arithmetic (an unevaluated sum hi + lo of two doubles, ~32 significant digits) built from
// the exact two-sum (Knuth) and the FMA two-product (Dekker), which holds the 18-point fits
// of the default context to far below the 1e-8 tolerance of the equation.
#include <cmath>
#include <cstdint>
#include <cstdio>

#include "common.cuh"

namespace cq {

namespace {

struct dd {
  double hi, lo;
};

__device__ __forceinline__ dd two_sum(double a, double b) {
  const double s = a + b, bb = s - a;
  return {s, (a - (s - bb)) + (b - bb)};
}
__device__ __forceinline__ dd quick_two_sum(double a, double b) {
  const double s = a + b;
  return {s, b - (s - a)};
}
__device__ __forceinline__ dd two_prod(double a, double b) {
  const double p = a * b;
  return {p, fma(a, b, -p)};
}
__device__ __forceinline__ dd mk_dd(double a) { return {a, 0.0}; }
__device__ __forceinline__ dd neg(dd a) { return {-a.hi, -a.lo}; }
__device__ __forceinline__ dd add(dd a, dd b) {
  dd s = two_sum(a.hi, b.hi);
  const dd t = two_sum(a.lo, b.lo);
  s.lo += t.hi;
  s = quick_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return quick_two_sum(s.hi, s.lo);
}
__device__ __forceinline__ dd sub(dd a, dd b) { return add(a, neg(b)); }
__device__ __forceinline__ dd mul(dd a, dd b) {
  dd p = two_prod(a.hi, b.hi);
  p.lo += a.hi * b.lo + a.lo * b.hi;
  return quick_two_sum(p.hi, p.lo);
}
// long division: three quotient digits, each corrected against the remainder
__device__ __forceinline__ dd div(dd a, dd b) {
  const double q1 = a.hi / b.hi;
  dd r = sub(a, mul(b, mk_dd(q1)));
  const double q2 = r.hi / b.hi;
  r = sub(r, mul(b, mk_dd(q2)));
  const double q3 = r.hi / b.hi;
  return add(quick_two_sum(q1, q2), mk_dd(q3));
}

struct cdd {
  dd re, im;
};
__device__ __forceinline__ cdd cadd(cdd a, cdd b) { return {add(a.re, b.re), add(a.im, b.im)}; }
__device__ __forceinline__ cdd csub(cdd a, cdd b) { return {sub(a.re, b.re), sub(a.im, b.im)}; }
__device__ __forceinline__ cdd cmul(cdd a, cdd b) {
  return {sub(mul(a.re, b.re), mul(a.im, b.im)), add(mul(a.re, b.im), mul(a.im, b.re))};
}
// a / b = a conj(b) / |b|^2
__device__ __forceinline__ cdd cdiv(cdd a, cdd b) {
  const dd den = add(mul(b.re, b.re), mul(b.im, b.im));
  const dd nr = add(mul(a.re, b.re), mul(a.im, b.im));
  const dd ni = sub(mul(a.im, b.re), mul(a.re, b.im));
  return {div(nr, den), div(ni, den)};
}

constexpr int kMaxFit = 64;

// Thiele coefficients a_i = g_i(z_i) of the points z_j = i w_j: g_0 = A, g_i(z_j) =
// (g_{i-1}(z_{i-1}) - g_{i-1}(z_j)) / ((z_j - z_{i-1}) g_{i-1}(z_j)), in place.
__device__ void pade_fit(const double* w, const double2* A, int64_t stride, int n, cdd* g) {
  for (int j = 0; j < n; ++j) g[j] = {mk_dd(A[(int64_t)j * stride].x), mk_dd(A[(int64_t)j * stride].y)};
  for (int i = 1; i < n; ++i) {
    const cdd gd = g[i - 1];
    for (int j = i; j < n; ++j) {
      const cdd dz = {mk_dd(0.0), sub(mk_dd(w[j]), mk_dd(w[i - 1]))};  // z_j - z_{i-1}
      g[j] = cdiv(csub(gd, g[j]), cmul(dz, g[j]));
    }
  }
}

// A(x + i y) from the coefficients: a_0 / (1 + a_1 (z - z_0) / (1 + a_2 (z - z_1) / ...))
__device__ double2 pade_eval(const double* w, const cdd* a, int n, double x, double y) {
  const cdd z = {mk_dd(x), mk_dd(y)};
  const cdd one = {mk_dd(1.0), mk_dd(0.0)};
  auto zmz = [&](int i) { return cdd{z.re, sub(z.im, mk_dd(w[i]))}; };
  cdd X = cmul(a[n - 1], zmz(n - 2));
  for (int f = 1; f < n - 1; ++f) {
    const int idx = n - f - 1;
    X = cdiv(cmul(a[idx], zmz(idx - 1)), cadd(one, X));
  }
  X = cdiv(a[0], cadd(one, X));
  return make_double2(X.re.hi + X.re.lo, X.im.hi + X.im.lo);
}

// method: 0 "sc" (bisection), 1 "sc_newton" (secant), 2 "linearized", 3 "spectral"
__global__ void k_qp_solve(const double* __restrict__ w, const double2* __restrict__ sigma,
                           const double* __restrict__ vhf, const double* __restrict__ e0,
                           int64_t nel, int n, double mu, double eta, double tol, int method,
                           double* __restrict__ e_out, double* __restrict__ res_out,
                           int* __restrict__ conv_out) {
  const int64_t I = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (I >= nel) return;
  cdd a[kMaxFit];
  pade_fit(w, sigma + I, nel, n, a);
  const double V = vhf[I], eps0 = e0[I];
  auto sig_re = [&](double x) { return pade_eval(w, a, n, x, eta).x; };
  auto res = [&](double e) { return e - V - sig_re(e - mu); };
  double E = eps0, R = 0.0;
  int conv = 1;
  if (method == 2) {  // linearised around eps0
    const double h = 1e-6;
    const double s0 = sig_re(eps0 - mu);
    const double ds = sig_re(eps0 - mu + h) - s0;
    const double Z = 1.0 / (1.0 - ds / h);
    E = Z * (V + s0 - (1.0 - 1.0 / Z) * eps0);
    R = res(E);
  } else if (method == 1) {  // secant from eps0
    double p0 = eps0, p1 = p0 >= 0 ? eps0 * (1 + 1e-4) + 1e-4 : eps0 * (1 + 1e-4) - 1e-4;
    double q0 = res(p0), q1 = res(p1), p = p1;
    if (fabs(q1) < fabs(q0)) {
      double t = p1; p1 = p0; p0 = t;
      t = q1; q1 = q0; q0 = t;
    }
    conv = 0;
    for (int it = 0; it < 400; ++it) {
      if (fabs(q1) > fabs(q0))
        p = (-q0 / q1 * p1 + p0) / (1 - q0 / q1);
      else
        p = (-q1 / q0 * p0 + p1) / (1 - q1 / q0);
      if (fabs(p - p1) < tol) {
        conv = 1;
        break;
      }
      p0 = p1;
      q0 = q1;
      p1 = p;
      q1 = res(p1);
    }
    E = p;
    R = res(p);
  } else if (method == 3) {  // the peak of the spectral function near eps0
    const int nw = 1000;
    const double wmin = eps0 - mu - 1.0, wmax = eps0 - mu + 1.0;
    double amax = 0.0, xbest = 0.0;
    int nmax = -1;
    for (int k = 0; k < nw; ++k) {
      const double x = wmin + k * (wmax - wmin) / (nw - 1);
      const double2 s = pade_eval(w, a, n, x, eta);
      const double gr = x + mu - V - s.x, gi = eta - s.y;  // 1 / (gr + i gi)
      const double A = fabs(gi / (gr * gr + gi * gi));
      if (A > amax) {
        amax = A;
        nmax = k;
        xbest = x;
      }
    }
    auto spec = [&](double x) {
      const double2 s = pade_eval(w, a, n, x, eta);
      const double gr = x + mu - V - s.x, gi = eta - s.y;
      return fabs(gi / (gr * gr + gi * gi));
    };
    if (nmax >= 0) {
      double step = tol, x = xbest, ax = spec(x + step);
      if (ax < amax) {
        step = -tol;
        ax = spec(x + step);
      }
      // climb while the peak rises; the maximum lies within one scan spacing of the best
      // grid point, which bounds the number of steps
      const long max_steps = (long)((wmax - wmin) / (nw - 1) / tol) + 2;
      for (long s = 0; ax >= amax && s < max_steps; ++s) {
        x += step;
        amax = ax;
        ax = spec(x + step);
      }
      E = x + mu;
    } else {
      E = eps0;
      conv = 0;
    }
    R = res(E);
  } else {  // bisection: bracket in steps of 0.01 from eps0, then halve
    double r = res(eps0);
    E = eps0;
    if (fabs(r) >= tol) {
      const double delta = 0.01;
      double e1, e2;
      int steps = 0;
      conv = 0;
      if (r >= 0) {
        e2 = eps0;
        e1 = eps0 - delta;
        double r1 = res(e1);
        while (r1 > 0 && steps++ < 100000) {
          e1 -= delta;
          r1 = res(e1);
        }
      } else {
        e1 = eps0;
        e2 = eps0 + delta;
        double r2 = res(e2);
        while (r2 < 0 && steps++ < 100000) {
          e2 += delta;
          r2 = res(e2);
        }
      }
      double em = 0.5 * (e1 + e2);
      r = res(em);
      for (int it = 0; it < 200 && fabs(r) > tol; ++it) {
        if (r >= 0)
          e2 = em;
        else
          e1 = em;
        em = 0.5 * (e1 + e2);
        r = res(em);
      }
      conv = fabs(r) <= tol;
      E = em;
    }
    R = r;
  }
  e_out[I] = E;
  res_out[I] = R;
  conv_out[I] = conv;
}

}  // namespace

void launch_qp_solve(const double* w, const double2* sigma, const double* vhf, const double* e0,
                     int64_t nel, int nfit, double mu, double eta, double tol, int method,
                     double* e_out, double* res_out, int* conv_out, cudaStream_t s) {
  CQ_REQUIRE(nfit >= 2 && nfit <= kMaxFit, COQUI_B200_EINVAL, "qp_solve: 2 <= Nfit <= 64");
  CQ_REQUIRE(method >= 0 && method <= 3, COQUI_B200_EINVAL, "qp_solve: unknown method");
  if (nel <= 0) return;
  k_qp_solve<<<(unsigned)((nel + 127) / 128), 128, 0, s>>>(w, sigma, vhf, e0, nel, nfit, mu, eta,
                                                           tol, method, e_out, res_out, conv_out);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
}

}  // namespace cq

extern "C" {

COQUI_B200_API int coqui_b200_qp_solve(const double* w_fit, const double* sigma_fit,
                                       const double* vhf, const double* e0, int64_t nel, int nfit,
                                       double mu, double eta, double tol, int method, int device,
                                       double* e_out, double* res_out, int* conv_out, char* errbuf,
                                       int errlen) {
  struct Bufs {
    void* p[7] = {};
    ~Bufs() {
      for (void* q : p)
        if (q) cudaFree(q);
    }
  } b;
  auto fail = [&](int code, const char* msg) {
    if (errbuf && errlen > 0) {
      std::snprintf(errbuf, (size_t)errlen, "%s", msg);
    }
    return code;
  };
  if (!w_fit || !sigma_fit || !vhf || !e0 || !e_out || !res_out || !conv_out)
    return fail(COQUI_B200_EINVAL, "qp_solve: null argument");
  if (nel < 0 || nfit < 2 || nfit > 64 || method < 0 || method > 3 || !(eta >= 0) || !(tol > 0))
    return fail(COQUI_B200_EINVAL, "qp_solve: bad argument (2 <= Nfit <= 64, method 0..3)");
  if (nel == 0) return COQUI_B200_OK;
  try {
    CQ_CHECK_CUDA(cudaSetDevice(device));
    const size_t sz[7] = {(size_t)nfit * 8, (size_t)nfit * nel * 16, (size_t)nel * 8,
                          (size_t)nel * 8, (size_t)nel * 8, (size_t)nel * 8, (size_t)nel * 4};
    for (int i = 0; i < 7; ++i) CQ_CHECK_CUDA(cudaMalloc(&b.p[i], sz[i]));
    CQ_CHECK_CUDA(cudaMemcpy(b.p[0], w_fit, sz[0], cudaMemcpyHostToDevice));
    CQ_CHECK_CUDA(cudaMemcpy(b.p[1], sigma_fit, sz[1], cudaMemcpyHostToDevice));
    CQ_CHECK_CUDA(cudaMemcpy(b.p[2], vhf, sz[2], cudaMemcpyHostToDevice));
    CQ_CHECK_CUDA(cudaMemcpy(b.p[3], e0, sz[3], cudaMemcpyHostToDevice));
    cq::launch_qp_solve((const double*)b.p[0], (const double2*)b.p[1], (const double*)b.p[2],
                        (const double*)b.p[3], nel, nfit, mu, eta, tol, method, (double*)b.p[4],
                        (double*)b.p[5], (int*)b.p[6], 0);
    CQ_CHECK_CUDA(cudaDeviceSynchronize());
    CQ_CHECK_CUDA(cudaMemcpy(e_out, b.p[4], sz[4], cudaMemcpyDeviceToHost));
    CQ_CHECK_CUDA(cudaMemcpy(res_out, b.p[5], sz[5], cudaMemcpyDeviceToHost));
    CQ_CHECK_CUDA(cudaMemcpy(conv_out, b.p[6], sz[6], cudaMemcpyDeviceToHost));
    return COQUI_B200_OK;
  } catch (const cq::Error& e) {
    return fail(e.code, e.what());
  }
}

}  // extern "C"
