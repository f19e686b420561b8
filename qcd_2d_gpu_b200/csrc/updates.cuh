// Staple gather and the three link updates.
//
// Staple of U_mu(x) in the plane (mu, nu), with the reference's product order
// (mc_updates.h:158-176 and the five sibling kernels):
//   forward   U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+
//   backward  U_nu(x+mu-nu)^+ U_mu(x-nu)^+ U_nu(x-nu)
// nu runs over (x, t) for mu = y, (y, t) for mu = x, (y, x) for mu = t, forward
// before backward, accumulated into a zero quaternion.  The boundary
// conditions are folded into the gather:
//   PCC  x and t links on the plane y = 0 are never updated
//        (mc_updates_pcc.h:29,83,134,189);
//   PMC  for mu = x, t the y staple that crosses y = Ly-1 <-> 0 is left out
//        (mc_updates_pmc.h:33,40,96,103,156,163,219,225); the y links
//        themselves use the periodic gather (mc_updates_pmc.h:250-251).
#pragma once
#include <curand_kernel.h>
#include "lattice.cuh"
#include "su2.cuh"

namespace qcd {

enum { KIND_METRO = 0, KIND_HB = 1, KIND_OR = 2 };

// device error word bits
// (DEVERR_TIMEOUT: a bounded wait of the wavefront or the fused-pair kernels ran out)
enum { DEVERR_HB_LOOP = 1, DEVERR_NONUNITARY = 2, DEVERR_TIMEOUT = 4 };

// The Kennedy-Pendleton rejection loop accepts with probability > 1/2 for any
// staple; this bound is only reached when the staple sum is zero or not
// finite, and then the update stops and flags the error instead of spinning.
#define QCD_HB_MAX_TRIES 4096

template <int MU>
struct Planes {
  static constexpr int NU1 = MU == DIR_Y ? DIR_X : DIR_Y;
  static constexpr int NU2 = MU == DIR_T ? DIR_X : DIR_T;
};

// FP32 staples add their second product straight into the sum with
// multiply-adds (A + X Y^+, A + X Y); FP64 keeps the reference's separate
// product and sum, whose rounding the bit-parity tests pin.
__device__ __forceinline__ Quat<float> q_acc_mul_bd(const Quat<float>& A, const Quat<float>& a, const Quat<float>& b) {
  Quat<float> c;
  c.w = A.w + a.w * b.w + a.x * b.x + a.y * b.y + a.z * b.z;
  c.x = A.x + a.x * b.w - a.w * b.x - a.y * b.z + a.z * b.y;
  c.y = A.y + a.y * b.w - a.z * b.x - a.w * b.y + a.x * b.z;
  c.z = A.z + a.z * b.w + a.y * b.x - a.w * b.z - a.x * b.y;
  return c;
}
__device__ __forceinline__ Quat<float> q_acc_mul(const Quat<float>& A, const Quat<float>& a, const Quat<float>& b) {
  Quat<float> c;
  c.w = A.w + a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z;
  c.x = A.x + a.x * b.w + a.w * b.x + a.y * b.z - a.z * b.y;
  c.y = A.y + a.y * b.w + a.z * b.x + a.w * b.y - a.x * b.z;
  c.z = A.z + a.z * b.w - a.y * b.x + a.w * b.z + a.x * b.y;
  return c;
}
__device__ __forceinline__ Quat<double> q_acc_mul_bd(const Quat<double>& A, const Quat<double>& a,
                                                     const Quat<double>& b) {
  return q_add(A, q_mul_bd(a, b));
}
__device__ __forceinline__ Quat<double> q_acc_mul(const Quat<double>& A, const Quat<double>& a, const Quat<double>& b) {
  return q_add(A, q_mul(a, b));
}

template <int MU, int NU, int BC, class L, class R>
__device__ __forceinline__ void add_staples(const L& links, const Geo& g, const Nbr& n, int par,
                                            Quat<R>& A) {
  const int o = par ^ 1;
  const bool drop_fwd = BC == BC_PMC && NU == DIR_Y && at_ytop(g, n);
  const bool drop_bwd = BC == BC_PMC && NU == DIR_Y && at_y0(g, n);
  if (!drop_fwd) {
    Quat<R> a = links.ld(NU, o, n.id + off_plus(n, MU));
    Quat<R> b = links.ld(MU, o, n.id + off_plus(n, NU));
    Quat<R> c = links.ld(NU, par, n.id);
    A = q_acc_mul_bd(A, q_mul_bd(a, b), c);
  }
  if (!drop_bwd) {
    const int m = n.id + off_minus(n, NU);
    Quat<R> a = links.ld(NU, par, m + off_plus(n, MU));
    Quat<R> b = links.ld(MU, o, m);
    Quat<R> c = links.ld(NU, o, m);
    A = q_acc_mul(A, q_mul_adbd(a, b), c);
  }
}

template <int MU, int BC, class L, class R>
__device__ __forceinline__ Quat<R> staple_sum(const L& links, const Geo& g, const Nbr& n, int par) {
  Quat<R> A = q_zero<R>();
  add_staples<MU, Planes<MU>::NU1, BC>(links, g, n, par, A);
  add_staples<MU, Planes<MU>::NU2, BC>(links, g, n, par, A);
  return A;
}

// ------------------------------------------------ FP64 (reference parity) --

// Kennedy-Pendleton heat-bath exactly as the reference draws and rounds it
// (mc_updates.h:43-64): float uniforms and float logf/cospif/sincospif for the
// distribution, the new link built in double and normalised with rsqrt.
// Returns the new link X A^+ with A the normalised staple.
__device__ __forceinline__ Quat<double> heatbath_ref(Quat<double> A, double beta,
                                                     curandStateMRG32k3a_t* st, int* err) {
  double a;
  A = q_normalize_norm(A, &a);
  float inv = (float)(0.5 / (a * beta)), lf, aux;
  for (int tries = 1;; tries++) {
    float r0 = curand_uniform(st), r1 = curand_uniform(st), r2 = curand_uniform(st);
    float c = cospif(2 * r1);
    lf = -(logf(r0) + c * c * logf(r2)) * inv;
    aux = 1 - curand_uniform(st);
    if (!(aux * aux > 1 - lf)) break;
    if (tries >= QCD_HB_MAX_TRIES) {
      atomicOr(err, DEVERR_HB_LOOP);
      break;
    }
  }
  Quat<double> X;
  X.w = 1 - 2 * (double)lf;
  double nrm = sqrt(1 - X.w * X.w);
  float ct = 2 * curand_uniform(st) - 1, sp, cp;
  sincospif(2 * curand_uniform(st), &sp, &cp);
  float stt = sqrtf(fmaxf(0.f, 1 - ct * ct));
  double v1 = ct, v2 = (double)stt * cp, v3 = (double)stt * sp;
  double s = nrm * rsqrt(v1 * v1 + v2 * v2 + v3 * v3);
  X.x = v1 * s;
  X.y = v2 * s;
  X.z = v3 * s;
  return q_mul_bd(X, A);
}

// exp(-s) > u decided in float unless u lies within 1e-4 (relative) of the
// float estimate, then in double (mc_updates.h:7-15).  Same decision as the
// double test.
__device__ __forceinline__ bool metropolis_accept(double s, double u) {
  const double tol = 1e-4;
  double ef = expf(-(float)s);
  if (u < ef * (1 - tol)) return true;
  if (u > ef * (1 + tol)) return false;
  return exp(-s) > u;
}

// `upd` Metropolis hits with proposals r U, r within eps of 1 (su2.h:87-97,
// mc_updates.h:16-36, 119-128); A (not normalised) is reused by every hit.
__device__ __forceinline__ int metropolis_ref(Quat<double>& U, const Quat<double>& A, double beta,
                                              double eps, int upd, curandStateMRG32k3a_t* st) {
  int acc = 0;
  for (int h = 0; h < upd; h++) {
    double r1 = curand_uniform_double(st) - 0.5;
    double r2 = curand_uniform_double(st) - 0.5;
    double r3 = curand_uniform_double(st) - 0.5;
    double nrm = sqrt(r1 * r1 + r2 * r2 + r3 * r3);
    Quat<double> r;
    r.x = eps * r1 / nrm;
    r.y = eps * r2 / nrm;
    r.z = eps * r3 / nrm;
    r.w = sqrt(1 - eps * eps);
    Quat<double> Un = q_mul(r, U);
    Quat<double> dU{Un.w - U.w, Un.x - U.x, Un.y - U.y, Un.z - U.z};
    double s = -beta * q_retr_mul(dU, A);
    bool ok = s < 0 ? true : metropolis_accept(s, curand_uniform_double(st));
    if (ok) {
      U = Un;
      acc++;
    }
  }
  return acc;
}

// U -> A^+ U^+ A^+ with A the normalised staple (mc_updates.h:109-115):
// leaves Re tr(U A) unchanged.
__device__ __forceinline__ Quat<double> overrelax_ref(Quat<double> A, const Quat<double>& U) {
  double a;
  A = q_normalize_norm(A, &a);
  Quat<double> B = q_mul_adbd(U, A);
  return q_mul_ad(A, B);
}

// ------------------------------------------- FP32 links + FP64 fix-ups ----
// The FP32 updates draw from a generator G with uniform() (float in (0, 1])
// and uniform_double() (double in (0, 1]): the counter-based PhiloxStream.

// Kennedy-Pendleton in FP32.  The accept test, which loses accuracy in single
// precision (1 - lf is within an ulp of 1 for large beta*|A|), is done in
// double.  The length of the spatial part is taken as n = 2 sqrt(lf (1 - lf))
// instead of sqrt(1 - X0^2): no cancellation as X0 -> 1, so float suffices.
// The draws come from the counter-based stream a whole block at a time: each
// try of the rejection loop takes one block (r0, r1, r2 and the accept
// uniform), the direction the first two words of the next one, the same
// words in the same order as drawing them one by one.
template <class G>
__device__ __forceinline__ Quat<float> heatbath_fast(Quat<float> A, float beta, G& st, int* err) {
  float det = q_det(A);
  float rinv = rsqrtf(det);
  float a = det * rinv;
  A = Quat<float>{A.w * rinv, A.x * rinv, A.y * rinv, A.z * rinv};
  float inv = 0.5f / (a * beta);
  float lf;
  uint32_t w[4];
  for (int tries = 1;; tries++) {
    st.block(w);
    const float r0 = G::u24(w[0]), r1 = G::u24(w[1]), r2 = G::u24(w[2]);
    // hardware approximations (absolute error ~2^-21): cos(2 pi r1) evaluated
    // as -cos(2 pi (r1 - 1/2)) keeps the argument in [-pi, pi]
    float c = -__cosf(6.2831853f * (r1 - 0.5f));
    lf = -(__logf(r0) + c * c * __logf(r2)) * inv;
    const float aux = 1.f - G::u24(w[3]);
    if (!((double)aux * aux > 1.0 - (double)lf)) break;
    if (tries >= QCD_HB_MAX_TRIES) {
      atomicOr(err, DEVERR_HB_LOOP);
      break;
    }
  }
  const float x0 = 1.f - 2.f * lf;
  const float nrm = 2.f * sqrtf(lf * (1.f - lf));
  st.block(w);
  float ct = 2.f * G::u24(w[0]) - 1.f, sp, cp;
  __sincosf(6.2831853f * (G::u24(w[1]) - 0.5f), &sp, &cp);  // angle + pi
  float stt = sqrtf(fmaxf(0.f, 1.f - ct * ct));
  Quat<float> X{x0, nrm * ct, -nrm * stt * cp, -nrm * stt * sp};
  return q_mul_bd(X, A);
}

// Over-relaxation U -> (Ahat U Ahat)^+, Ahat = A/|A| (mc_updates.h:109-115),
// written with the quaternion identity q p q = 2 <q, pbar> q - |q|^2 pbar:
//   U' = 2 (<A, Ubar> / |A|^2) Abar - U,   <A, Ubar> = 1/2 Re tr(U A),
// the same map as the reference's two products with ~16 operations instead of
// ~41; it keeps <A, Ubar> (the local action) and |U'| = |U| exactly in exact
// arithmetic.  FP32 only: the FP64 path keeps the reference's products.
__device__ __forceinline__ Quat<float> overrelax_fast(const Quat<float>& A, const Quat<float>& U) {
  const float c = __fdividef(2.f * q_retr_mul(A, U), q_det(A));
  return Quat<float>{c * A.w - U.w, -c * A.x - U.x, -c * A.y - U.y, -c * A.z - U.z};
}

// Metropolis with FP32 links: proposal and action change in float, the
// accept decision with the same single-then-double test as the reference.
template <class G>
__device__ __forceinline__ int metropolis_fast(Quat<float>& U, const Quat<float>& A, float beta,
                                               float eps, int upd, G& st) {
  int acc = 0;
  const float r0 = sqrtf(1.f - eps * eps);
  for (int h = 0; h < upd; h++) {
    float r1 = st.uniform() - 0.5f;
    float r2 = st.uniform() - 0.5f;
    float r3 = st.uniform() - 0.5f;
    float sc = eps * rsqrtf(r1 * r1 + r2 * r2 + r3 * r3);
    Quat<float> r{r0, sc * r1, sc * r2, sc * r3};
    Quat<float> Un = q_mul(r, U);
    Quat<float> dU{Un.w - U.w, Un.x - U.x, Un.y - U.y, Un.z - U.z};
    double s = -(double)beta * (double)q_retr_mul(dU, A);
    bool ok = s < 0 ? true : metropolis_accept(s, st.uniform_double());
    if (ok) {
      U = Un;
      acc++;
    }
  }
  return acc;
}

// Re-projection of an FP32 link with the norm taken in double.
__device__ __forceinline__ Quat<float> renorm_fast(const Quat<float>& u) {
  double d = (double)u.w * u.w + (double)u.x * u.x + (double)u.y * u.y + (double)u.z * u.z;
  double inv = rsqrt(d);
  return Quat<float>{(float)(u.w * inv), (float)(u.x * inv), (float)(u.y * inv),
                     (float)(u.z * inv)};
}

}  // namespace qcd
