/*
 * CPU oracle for the checkerboard SU(2) Wilson-action sweep — TEST
 * INFRASTRUCTURE, never part of the product (see oracle.h).
 *
 * Restates, on the reference's own AoS FP64 layout:
 *   su2 algebra ............ functions/su2.h:1-97
 *   heat_bath .............. functions/mc_updates.h:43-64
 *   metropolis(+accept) .... functions/mc_updates.h:7-36, su2.h:87-97
 *   over_relaxation ........ functions/mc_updates.h:109-115
 *   six phase kernels ...... functions/mc_updates.h:129-465 (periodic),
 *                            mc_updates_pcc.h:4-214, mc_updates_pmc.h:4-247
 *   sweep order ............ mc_updates.h:467-475, _pcc.h:216-224, _pmc.h:249-257
 *   starts ................. lattice_setup.h:24-81
 *   normalize .............. lattice_setup.h:202-207
 *   en_av .................. observables.h:1-21, 99-141
 *
 * Floating point: built with -ffp-contract=off, so every operation rounds
 * exactly as written.  nvcc contracts a*b+c into an FMA; the two places where
 * that changes a FLOAT result of the heat-bath are written with fmaf here
 * (ORA_FMA_LF, ORA_FMA_ST; pinned against the reference's outputs).  Double
 * contractions and CUDA's rsqrt (within 1 ulp of 1/sqrt) move results by
 * ~1e-16, far inside the 1e-12 parity bound.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef ORA_FMA_LF
#define ORA_FMA_LF 1
#endif
#ifndef ORA_FMA_ST
#define ORA_FMA_ST 1
#endif

typedef struct {
  double w, x, y, z;
} quat;

/* ---------------------------------------------------------------- MRG32k3a
 * L'Ecuyer (1999), "Good parameters and implementations for combined multiple
 * recursive random number generators", Operations Research 47(1):
 *   x_n = (1403580 x_{n-2} - 810728 x_{n-3}) mod 4294967087
 *   y_n = (527612 y_{n-1} - 1370589 y_{n-3}) mod 4294944443
 *   u_n = ((x_n - y_n) mod m1) / (m1 + 1), with 0 mapped to m1 / (m1 + 1).
 * Streams are 2^127 steps apart (RngStreams, L'Ecuyer et al. 2002); the jump
 * matrices are computed here by repeated squaring. */
#define MRG_M1 4294967087LL
#define MRG_M2 4294944443LL
#define MRG_NORM 2.328306549295727688e-10

typedef struct {
  int64_t s1[3], s2[3];
} mrg_state;

static double mrg_next(mrg_state* g) {
  int64_t p1 = (1403580LL * g->s1[1] - 810728LL * g->s1[0]) % MRG_M1;
  if (p1 < 0) p1 += MRG_M1;
  g->s1[0] = g->s1[1];
  g->s1[1] = g->s1[2];
  g->s1[2] = p1;
  int64_t p2 = (527612LL * g->s2[2] - 1370589LL * g->s2[0]) % MRG_M2;
  if (p2 < 0) p2 += MRG_M2;
  g->s2[0] = g->s2[1];
  g->s2[1] = g->s2[2];
  g->s2[2] = p2;
  return p1 > p2 ? (double)(p1 - p2) * MRG_NORM : (double)(p1 - p2 + MRG_M1) * MRG_NORM;
}

typedef struct {
  uint64_t a[3][3];
} mat3;

static mat3 mat_mul(const mat3* x, const mat3* y, uint64_t m) {
  mat3 r;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      unsigned __int128 s = 0;
      for (int k = 0; k < 3; k++) s += (unsigned __int128)x->a[i][k] * y->a[k][j];
      r.a[i][j] = (uint64_t)(s % m);
    }
  return r;
}

static void mat_vec(const mat3* x, int64_t v[3], uint64_t m) {
  int64_t r[3];
  for (int i = 0; i < 3; i++) {
    unsigned __int128 s = 0;
    for (int k = 0; k < 3; k++) s += (unsigned __int128)x->a[i][k] * (uint64_t)v[k];
    r[i] = (int64_t)(s % m);
  }
  memcpy(v, r, sizeof(r));
}

#define JUMP_BITS 40
static mat3 g_jump1[JUMP_BITS], g_jump2[JUMP_BITS];
static int g_jumps_ready = 0;

static void make_jumps(void) {
  if (g_jumps_ready) return;
  mat3 a1 = {{{0, 1, 0}, {0, 0, 1}, {(uint64_t)(MRG_M1 - 810728), 1403580, 0}}};
  mat3 a2 = {{{0, 1, 0}, {0, 0, 1}, {(uint64_t)(MRG_M2 - 1370589), 0, 527612}}};
  for (int i = 0; i < 127; i++) { /* A^(2^127) */
    a1 = mat_mul(&a1, &a1, MRG_M1);
    a2 = mat_mul(&a2, &a2, MRG_M2);
  }
  for (int b = 0; b < JUMP_BITS; b++) {
    g_jump1[b] = a1;
    g_jump2[b] = a2;
    a1 = mat_mul(&a1, &a1, MRG_M1);
    a2 = mat_mul(&a2, &a2, MRG_M2);
  }
  g_jumps_ready = 1;
}

static void mrg_stream(mrg_state* g, unsigned long long seed, long long id) {
  g->s1[0] = 12345 + (int64_t)(seed % (unsigned long long)(MRG_M1 - 12345));
  g->s1[1] = g->s1[2] = 12345;
  g->s2[0] = 12345 + (int64_t)(seed % (unsigned long long)(MRG_M2 - 12345));
  g->s2[1] = g->s2[2] = 12345;
  for (int b = 0; b < JUMP_BITS; b++)
    if ((id >> b) & 1) {
      mat_vec(&g_jump1[b], g->s1, MRG_M1);
      mat_vec(&g_jump2[b], g->s2, MRG_M2);
    }
}

/* ------------------------------------------------------------ handle ---- */
struct ora_lattice {
  ora_params p;
  int lyh, slice, vh;
  long long V;
  double* phi; /* V*12, reference layout */
  int* accept; /* V */
  const ora_tape_record* tape;
  int tape_streams, tape_draws;
  int* cursor;     /* tape: next draw per stream */
  mrg_state* own;  /* own generator per stream */
  long long* used; /* draws consumed per stream */
  volatile int err;
};

typedef struct {
  double ud;
  float uf;
  long long idx; /* tape record index, -1 for OWN */
} draw_t;

static inline draw_t draw(ora_lattice* h, int sid) {
  draw_t d;
  h->used[sid]++;
  if (h->tape) {
    int k = h->cursor[sid]++;
    if (k >= h->tape_draws) {
      h->err = ORA_ERR_TAPE;
      d.ud = 0.5;
      d.uf = 0.5f;
      d.idx = -2;
      return d;
    }
    long long i = (long long)sid * h->tape_draws + k;
    d.ud = h->tape[i].ud;
    d.uf = h->tape[i].uf;
    d.idx = i;
    return d;
  }
  d.ud = mrg_next(&h->own[sid]);
  d.uf = (float)d.ud;
  d.idx = -1;
  return d;
}

static inline float f_log(const ora_lattice* h, draw_t d) {
  return d.idx >= 0 ? h->tape[d.idx].log_uf : logf(d.uf);
}
static inline float f_cospi2(const ora_lattice* h, draw_t d) {
  return d.idx >= 0 ? h->tape[d.idx].cospi_2uf : (float)cos(2.0 * M_PI * (double)d.uf);
}
static inline void f_sincospi2(const ora_lattice* h, draw_t d, float* s, float* c) {
  if (d.idx >= 0) {
    *s = h->tape[d.idx].sc_sin;
    *c = h->tape[d.idx].sc_cos;
  } else {
    *s = (float)sin(2.0 * M_PI * (double)d.uf);
    *c = (float)cos(2.0 * M_PI * (double)d.uf);
  }
}

/* ------------------------------------------------------------ su2.h ----- */
static inline quat q_ld(const double* p) { return (quat){p[0], p[1], p[2], p[3]}; }
static inline void q_st(double* p, quat u) {
  p[0] = u.w;
  p[1] = u.x;
  p[2] = u.y;
  p[3] = u.z;
}
static inline quat q_add(quat a, quat b) { return (quat){a.w + b.w, a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline quat q_mul(quat a, quat b) { /* su2.h:50-55 */
  quat c;
  c.w = a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z;
  c.x = a.x * b.w + a.w * b.x + a.y * b.z - a.z * b.y;
  c.y = a.y * b.w + a.z * b.x + a.w * b.y - a.x * b.z;
  c.z = a.z * b.w - a.y * b.x + a.w * b.z + a.x * b.y;
  return c;
}
static inline quat q_mul_bd(quat a, quat b) { /* A B^+, su2.h:56-61 */
  quat c;
  c.w = a.w * b.w + a.x * b.x + a.y * b.y + a.z * b.z;
  c.x = a.x * b.w - a.w * b.x - a.y * b.z + a.z * b.y;
  c.y = a.y * b.w - a.z * b.x - a.w * b.y + a.x * b.z;
  c.z = a.z * b.w + a.y * b.x - a.w * b.z - a.x * b.y;
  return c;
}
static inline quat q_mul_ad(quat a, quat b) { /* A^+ B, su2.h:62-67 */
  quat c;
  c.w = a.w * b.w + a.x * b.x + a.y * b.y + a.z * b.z;
  c.x = -a.x * b.w + a.w * b.x - a.y * b.z + a.z * b.y;
  c.y = -a.y * b.w - a.z * b.x + a.w * b.y + a.x * b.z;
  c.z = -a.z * b.w + a.y * b.x + a.w * b.z - a.x * b.y;
  return c;
}
static inline quat q_mul_adbd(quat a, quat b) { /* A^+ B^+, su2.h:68-73 */
  quat c;
  c.w = a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z;
  c.x = -a.x * b.w - a.w * b.x + a.y * b.z - a.z * b.y;
  c.y = -a.y * b.w + a.z * b.x - a.w * b.y - a.x * b.z;
  c.z = -a.z * b.w - a.y * b.x - a.w * b.z + a.x * b.y;
  return c;
}
static inline double q_det(quat a) { return a.w * a.w + a.x * a.x + a.y * a.y + a.z * a.z; }
static inline quat q_scale(quat a, double s) { return (quat){a.w * s, a.x * s, a.y * s, a.z * s}; }
static inline quat q_normalize(quat a) { return q_scale(a, 1.0 / sqrt(q_det(a))); } /* su2.h:4-8 */

/* ------------------------------------------------------ link updates ---- */
/* Kennedy-Pendleton, mc_updates.h:43-64 */
static quat heat_bath(ora_lattice* h, int sid, quat A) {
  double det = q_det(A), inv = 1.0 / sqrt(det); /* su2_normalize_det, su2.h:16-21 */
  A = q_scale(A, inv);
  double a = det * inv;
  float finv = (float)(0.5 / (a * (double)h->p.beta)), lf = 0.f, aux;
  for (int tries = 0; tries < 4096; tries++) {
    draw_t d0 = draw(h, sid), d1 = draw(h, sid), d2 = draw(h, sid);
    float c = f_cospi2(h, d1);
    float l0 = f_log(h, d0), l2 = f_log(h, d2);
    float cc = c * c;
#if ORA_FMA_LF
    float sum = fmaf(cc, l2, l0);
#else
    float sum = l0 + cc * l2;
#endif
    lf = -sum * finv;
    aux = 1 - draw(h, sid).uf;
    if (!(aux * aux > 1 - lf)) break;
  }
  quat X;
  X.w = 1 - 2 * (double)lf;
  double nrm = sqrt(1 - X.w * X.w);
  float ct = 2 * draw(h, sid).uf - 1, sp, cp;
  f_sincospi2(h, draw(h, sid), &sp, &cp);
#if ORA_FMA_ST
  float one_m = fmaf(-ct, ct, 1.0f);
#else
  float one_m = 1 - ct * ct;
#endif
  float stt = sqrtf(fmaxf(0.f, one_m));
  double v1 = ct, v2 = (double)stt * cp, v3 = (double)stt * sp;
  double s = nrm * (1.0 / sqrt(v1 * v1 + v2 * v2 + v3 * v3));
  X.x = v1 * s;
  X.y = v2 * s;
  X.z = v3 * s;
  return q_mul_bd(X, A);
}

/* mc_updates.h:7-15 */
static int metropolis_accept(double s, double u) {
  const double tol = 1e-4;
  double ef = expf(-(float)s);
  if (u < ef * (1 - tol)) return 1;
  if (u > ef * (1 + tol)) return 0;
  return exp(-s) > u;
}

/* mc_updates.h:16-36 with su2_update su2.h:87-97, `upd` hits (mc_updates.h:123-126) */
static int metropolis(ora_lattice* h, int sid, quat* U, quat A) {
  const double beta = (double)h->p.beta, eps = (double)h->p.epsilon;
  int acc = 0;
  for (int hit = 0; hit < h->p.upd; hit++) {
    double r1 = draw(h, sid).ud - 0.5;
    double r2 = draw(h, sid).ud - 0.5;
    double r3 = draw(h, sid).ud - 0.5;
    double n = sqrt(r1 * r1 + r2 * r2 + r3 * r3);
    quat r = {sqrt(1 - eps * eps), eps * r1 / n, eps * r2 / n, eps * r3 / n};
    quat Un = q_mul(r, *U);
    quat dU = {Un.w - U->w, Un.x - U->x, Un.y - U->y, Un.z - U->z};
    double s = -beta * (dU.w * A.w - dU.x * A.x - dU.y * A.y - dU.z * A.z);
    int ok = s < 0 ? 1 : metropolis_accept(s, draw(h, sid).ud);
    if (ok) {
      *U = Un;
      acc++;
    }
  }
  return acc;
}

/* mc_updates.h:109-115 */
static quat over_relaxation(quat A, quat U) {
  A = q_normalize(A);
  return q_mul_ad(A, q_mul_adbd(U, A));
}

/* ------------------------------------------------------------- phases --- */
/* Offsets, in half-lattice sites, of the six neighbours of half-lattice site
 * id on sublattice `par` (all on the other sublattice); see
 * mc_updates.h:139-153 for the even and :195-210 for the odd form. */
typedef struct {
  int yq, x, t, q, yp, ym, xp, xm, tp, tm;
} nbr_t;

static inline nbr_t nbr(const ora_lattice* h, int id, int par) {
  nbr_t n;
  n.yq = id % h->lyh;
  int r = id / h->lyh;
  n.x = r % h->p.lx;
  n.t = r / h->p.lx;
  n.q = ((n.t + n.x) & 1) ^ par; /* parity of the physical y */
  n.yp = n.q ? (n.yq == h->lyh - 1 ? -(h->lyh - 1) : 1) : 0;
  n.ym = n.q ? 0 : (n.yq == 0 ? h->lyh - 1 : -1);
  n.xp = n.x == h->p.lx - 1 ? -(h->p.lx - 1) * h->lyh : h->lyh;
  n.xm = n.x == 0 ? (h->p.lx - 1) * h->lyh : -h->lyh;
  n.tp = n.t == h->p.lt - 1 ? -(h->p.lt - 1) * h->slice : h->slice;
  n.tm = n.t == 0 ? (h->p.lt - 1) * h->slice : -h->slice;
  return n;
}

static inline int plus(const nbr_t* n, int d) { return d == 0 ? n->yp : d == 1 ? n->xp : n->tp; }
static inline int minus(const nbr_t* n, int d) { return d == 0 ? n->ym : d == 1 ? n->xm : n->tm; }

/* link d of half-lattice site j on sublattice par */
static inline double* L(const ora_lattice* h, int par, int j, int d) {
  return h->phi + ((size_t)par * h->vh + j) * 12 + d * 4;
}

static quat staples(const ora_lattice* h, int mu, int par, int id, const nbr_t* n) {
  const int o = par ^ 1;
  const int nus[3][2] = {{1, 2}, {0, 2}, {0, 1}}; /* y:(x,t) x:(y,t) t:(y,x) */
  quat A = {0, 0, 0, 0};
  for (int k = 0; k < 2; k++) {
    int nu = nus[mu][k];
    int pmc = h->p.boundary == 2 && nu == 0; /* mc_updates_pmc.h:33,40 */
    int drop_fwd = pmc && n->yq == h->lyh - 1 && n->q == 1;
    int drop_bwd = pmc && n->yq == 0 && n->q == 0;
    if (!drop_fwd) {
      quat a = q_ld(L(h, o, id + plus(n, mu), nu));
      quat b = q_ld(L(h, o, id + plus(n, nu), mu));
      quat c = q_ld(L(h, par, id, nu));
      A = q_add(A, q_mul_bd(q_mul_bd(a, b), c));
    }
    if (!drop_bwd) {
      int m = id + minus(n, nu);
      quat a = q_ld(L(h, par, m + plus(n, mu), nu));
      quat b = q_ld(L(h, o, m, mu));
      quat c = q_ld(L(h, o, m, nu));
      A = q_add(A, q_mul(q_mul_adbd(a, b), c));
    }
  }
  return A;
}

int ora_phase(ora_lattice* h, int k, int kind) {
  if (!h || k < 0 || k > 5 || kind < 0 || kind > 2) return ORA_ERR_INVALID;
  const int mu = k / 2, par = k % 2;
#pragma omp parallel for schedule(static)
  for (int id = 0; id < h->vh; id++) {
    nbr_t n = nbr(h, id, par);
    /* PCC: x,t links at y = 0 stay fixed (mc_updates_pcc.h:29,83,134,189) */
    if (h->p.boundary == 1 && mu != 0 && n.yq == 0 && n.q == 0) continue;
    quat A = staples(h, mu, par, id, &n);
    double* u = L(h, par, id, mu);
    size_t site = (size_t)par * h->vh + id;
    if (kind == 1) {
      q_st(u, heat_bath(h, id, A));
      h->accept[site] += 1;
    } else if (kind == 0) {
      quat U = q_ld(u);
      h->accept[site] += metropolis(h, id, &U, A);
      q_st(u, U);
    } else {
      q_st(u, over_relaxation(A, q_ld(u)));
      h->accept[site] += 1;
    }
  }
  return h->err;
}

int ora_sweep(ora_lattice* h, int n) {
  if (!h) return ORA_ERR_INVALID;
  for (int s = 0; s < n; s++)
    for (int k = 0; k < 6; k++) {
      int rc = ora_phase(h, k, h->p.algo == 1 ? 1 : 0);
      if (rc) return rc;
    }
  return ORA_OK;
}

int ora_overrelax(ora_lattice* h, int n) {
  if (!h) return ORA_ERR_INVALID;
  for (int s = 0; s < n; s++)
    for (int k = 0; k < 6; k++) {
      int rc = ora_phase(h, k, 2);
      if (rc) return rc;
    }
  return ORA_OK;
}

/* --------------------------------------------------------- starts ------- */
int ora_init_cold(ora_lattice* h) { /* id_init2, lattice_setup.h:38-51 */
  if (!h) return ORA_ERR_INVALID;
  for (long long s = 0; s < h->V * 3; s++) q_st(h->phi + s * 4, (quat){1, 0, 0, 0});
  return ORA_OK;
}

int ora_init_hot(ora_lattice* h) { /* rand_init2(_pcc), lattice_setup.h:24-37,52-81 */
  if (!h) return ORA_ERR_INVALID;
#pragma omp parallel for schedule(static)
  for (int id = 0; id < h->vh; id++)
    for (int par = 0; par < 2; par++) {
      nbr_t n = nbr(h, id, par);
      int frozen = h->p.boundary == 1 && n.yq == 0 && n.q == 0;
      for (int d = 0; d < 3; d++) {
        quat a;
        if (d != 0 && frozen) {
          a = (quat){1, 0, 0, 0};
        } else {
          a.w = draw(h, id).ud - 0.5; /* su2_rand, su2.h:29-34 */
          a.x = draw(h, id).ud - 0.5;
          a.y = draw(h, id).ud - 0.5;
          a.z = draw(h, id).ud - 0.5;
          a = q_normalize(a);
        }
        q_st(L(h, par, id, d), a);
      }
    }
  return h->err;
}

int ora_load(ora_lattice* h, const double* aos) {
  if (!h || !aos) return ORA_ERR_INVALID;
  memcpy(h->phi, aos, (size_t)h->V * 12 * sizeof(double));
  return ORA_OK;
}

int ora_normalize(ora_lattice* h) { /* lattice_setup.h:202-207 */
  if (!h) return ORA_ERR_INVALID;
  for (long long s = 0; s < h->V * 3; s++) q_st(h->phi + s * 4, q_normalize(q_ld(h->phi + s * 4)));
  return ORA_OK;
}

/* ------------------------------------------------------- measurement ---- */
/* 1 - 1/2 Re tr U_mu(x) U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+  (observables.h:1-21) */
static double plaq(const ora_lattice* h, int par, int id, int mu, int nu, int omu, int onu) {
  quat A = q_mul(q_ld(L(h, par, id, mu)), q_ld(L(h, par ^ 1, id + omu, nu)));
  quat B = q_mul_bd(A, q_ld(L(h, par ^ 1, id + onu, mu)));
  A = q_mul_bd(B, q_ld(L(h, par, id, nu)));
  return 1 - A.w;
}

int ora_measure(ora_lattice* h, double* energy, double* plaquette) { /* observables.h:99-141 */
  if (!h) return ORA_ERR_INVALID;
  double e = 0, pl = 0;
  for (int par = 0; par < 2; par++)
    for (int id = 0; id < h->vh; id++) {
      nbr_t n = nbr(h, id, par);
      double a = plaq(h, par, id, 0, 1, n.yp, n.xp);
      double b = plaq(h, par, id, 0, 2, n.yp, n.tp);
      double c = plaq(h, par, id, 1, 2, n.xp, n.tp);
      if (h->p.boundary == 2 && n.yq == h->lyh - 1 && n.q == 1) a = b = 0;
      e += -c;
      pl += (3 - a - b - c) / 3;
    }
  if (energy) *energy = e / (double)h->V;
  if (plaquette) *plaquette = pl / (double)h->V;
  return ORA_OK;
}

/* -------------------------------------------------------- lifecycle ----- */
ora_lattice* ora_create(const ora_params* p, const ora_tape_record* tape, int tape_streams,
                        int tape_draws) {
  if (!p || p->lt < 2 || p->lx < 2 || p->ly < 2 || (p->lt | p->lx | p->ly) & 1) return NULL;
  if (p->algo < 0 || p->algo > 1 || p->boundary < 0 || p->boundary > 2) return NULL;
  ora_lattice* h = (ora_lattice*)calloc(1, sizeof(ora_lattice));
  if (!h) return NULL;
  h->p = *p;
  h->lyh = p->ly / 2;
  h->slice = h->lyh * p->lx;
  h->V = (long long)p->lt * p->lx * p->ly;
  h->vh = (int)(h->V / 2);
  h->phi = (double*)calloc((size_t)h->V * 12, sizeof(double));
  h->accept = (int*)calloc((size_t)h->V, sizeof(int));
  h->used = (long long*)calloc((size_t)h->vh, sizeof(long long));
  if (!h->phi || !h->accept || !h->used) goto fail;
  if (tape) {
    if (tape_streams < h->vh || tape_draws <= 0) goto fail;
    h->tape = tape;
    h->tape_streams = tape_streams;
    h->tape_draws = tape_draws;
    h->cursor = (int*)calloc((size_t)h->vh, sizeof(int));
    if (!h->cursor) goto fail;
  } else {
    make_jumps();
    h->own = (mrg_state*)malloc((size_t)h->vh * sizeof(mrg_state));
    if (!h->own) goto fail;
#pragma omp parallel for schedule(static)
    for (int id = 0; id < h->vh; id++) mrg_stream(&h->own[id], p->seed, id);
  }
  return h;
fail:
  ora_destroy(h);
  return NULL;
}

void ora_destroy(ora_lattice* h) {
  if (!h) return;
  free(h->phi);
  free(h->accept);
  free(h->used);
  free(h->cursor);
  free(h->own);
  free(h);
}

const double* ora_field(const ora_lattice* h) { return h ? h->phi : NULL; }
const int* ora_accept(const ora_lattice* h) { return h ? h->accept : NULL; }
long long ora_volume(const ora_lattice* h) { return h ? h->V : 0; }

long long ora_max_draws(const ora_lattice* h) {
  long long m = 0;
  if (!h) return 0;
  for (int i = 0; i < h->vh; i++)
    if (h->used[i] > m) m = h->used[i];
  return m;
}

int ora_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

int ora_get_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ================================================ FP32 links + FP64 fix-ups
 * Restatement of the library's own FP32 update path, the checker of its FP32
 * kernels (heatbath_fast, metropolis_fast, overrelax_fast and renorm_fast in
 * qcd_2d_gpu_b200/csrc/updates.cuh, site32 in csrc/sites.cuh).  The reference
 * has FP64 links only; its algorithm (mc_updates.h:7-64,109-115 and the PCC/PMC
 * masks of mc_updates_pcc.h / mc_updates_pmc.h) is kept step for step, with the
 * arithmetic in float except for the fix-ups done in double: the heat-bath
 * accept test, the Metropolis action change and accept test, and the
 * re-projection.
 *
 * The field holds float values (as doubles): links are read as floats and
 * written back as (double)float.  Draws come from Philox4x32-10 (Salmon,
 * Moraes, Dror, Shaw, SC'11) with counter (site, block, phase lo, phase hi)
 * and key (seed lo, seed hi), consumed word by word.  Host libm stands in for
 * the GPU's hardware cos/log/sincos (absolute error ~2^-21 there), so a
 * heat-bath accept decision can come out differently in rare cases; the
 * checks compare at float tolerance and count such sites. */
typedef struct {
  float w, x, y, z;
} fquat;

static inline fquat f_ld(const double* p) { return (fquat){(float)p[0], (float)p[1], (float)p[2], (float)p[3]}; }
static inline void f_st(double* p, fquat u) {
  p[0] = u.w;
  p[1] = u.x;
  p[2] = u.y;
  p[3] = u.z;
}
static inline fquat f_add(fquat a, fquat b) { return (fquat){a.w + b.w, a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline fquat f_mul(fquat a, fquat b) { /* su2.h:50-55 in float */
  fquat c;
  c.w = a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z;
  c.x = a.x * b.w + a.w * b.x + a.y * b.z - a.z * b.y;
  c.y = a.y * b.w + a.z * b.x + a.w * b.y - a.x * b.z;
  c.z = a.z * b.w - a.y * b.x + a.w * b.z + a.x * b.y;
  return c;
}
static inline fquat f_mul_bd(fquat a, fquat b) { /* su2.h:56-61 */
  fquat c;
  c.w = a.w * b.w + a.x * b.x + a.y * b.y + a.z * b.z;
  c.x = a.x * b.w - a.w * b.x - a.y * b.z + a.z * b.y;
  c.y = a.y * b.w - a.z * b.x - a.w * b.y + a.x * b.z;
  c.z = a.z * b.w + a.y * b.x - a.w * b.z - a.x * b.y;
  return c;
}
static inline fquat f_mul_ad(fquat a, fquat b) { /* su2.h:62-67 */
  fquat c;
  c.w = a.w * b.w + a.x * b.x + a.y * b.y + a.z * b.z;
  c.x = -a.x * b.w + a.w * b.x - a.y * b.z + a.z * b.y;
  c.y = -a.y * b.w - a.z * b.x + a.w * b.y + a.x * b.z;
  c.z = -a.z * b.w + a.y * b.x + a.w * b.z - a.x * b.y;
  return c;
}
static inline fquat f_mul_adbd(fquat a, fquat b) { /* su2.h:68-73 */
  fquat c;
  c.w = a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z;
  c.x = -a.x * b.w - a.w * b.x + a.y * b.z - a.z * b.y;
  c.y = -a.y * b.w + a.z * b.x - a.w * b.y - a.x * b.z;
  c.z = -a.z * b.w - a.y * b.x - a.w * b.z + a.x * b.y;
  return c;
}
static inline float f_det(fquat a) { return a.w * a.w + a.x * a.x + a.y * a.y + a.z * a.z; }
static inline fquat f_scale(fquat a, float s) { return (fquat){a.w * s, a.x * s, a.y * s, a.z * s}; }

/* Philox4x32-10: ten rounds of two 32 x 32 -> 64-bit products with the
 * multipliers 0xD2511F53 and 0xCD9E8D57, the round key bumped by the Weyl
 * increments 0x9E3779B9 and 0xBB67AE85 between rounds. */
static void philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t x0 = ctr[0], x1 = ctr[1], x2 = ctr[2], x3 = ctr[3], k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; r++) {
    if (r) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    uint64_t p0 = (uint64_t)0xD2511F53u * x0, p1 = (uint64_t)0xCD9E8D57u * x2;
    uint32_t y0 = (uint32_t)(p1 >> 32) ^ x1 ^ k0, y2 = (uint32_t)(p0 >> 32) ^ x3 ^ k1;
    x1 = (uint32_t)p1;
    x3 = (uint32_t)p0;
    x0 = y0;
    x2 = y2;
  }
  out[0] = x0;
  out[1] = x1;
  out[2] = x2;
  out[3] = x3;
}

typedef struct {
  uint32_t ctr[4], key[2], buf[4];
  int left, pos;
} pstream;

static inline void ps_init(pstream* s, unsigned long long seed, uint32_t site, unsigned long long phase) {
  s->key[0] = (uint32_t)seed;
  s->key[1] = (uint32_t)(seed >> 32);
  s->ctr[0] = site;
  s->ctr[1] = 0;
  s->ctr[2] = (uint32_t)phase;
  s->ctr[3] = (uint32_t)(phase >> 32);
  s->left = 0;
  s->pos = 0;
}
static inline uint32_t ps_next(pstream* s) {
  if (s->left == 0) {
    philox4x32_10(s->ctr, s->key, s->buf);
    s->ctr[1]++;
    s->left = 4;
    s->pos = 0;
  }
  s->left--;
  return s->buf[s->pos++];
}
/* (k + 1) / 2^24 of the top 24 bits: a float in (0, 1] */
static inline float ps_uniform(pstream* s) { return (float)((ps_next(s) >> 8) + 1u) * 5.9604644775390625e-8f; }
/* (k + 1) / 2^53 of 53 bits of two words: a double in (0, 1] */
static inline double ps_uniform_double(pstream* s) {
  uint64_t hi = ps_next(s), lo = ps_next(s);
  return (double)(((hi << 21) | (lo >> 11)) + 1ull) * 1.1102230246251565e-16;
}

static fquat staples32(const ora_lattice* h, int mu, int par, int id, const nbr_t* n) {
  const int o = par ^ 1;
  const int nus[3][2] = {{1, 2}, {0, 2}, {0, 1}};
  fquat A = {0, 0, 0, 0};
  for (int k = 0; k < 2; k++) {
    int nu = nus[mu][k];
    int pmc = h->p.boundary == 2 && nu == 0;
    int drop_fwd = pmc && n->yq == h->lyh - 1 && n->q == 1;
    int drop_bwd = pmc && n->yq == 0 && n->q == 0;
    if (!drop_fwd) {
      fquat a = f_ld(L(h, o, id + plus(n, mu), nu));
      fquat b = f_ld(L(h, o, id + plus(n, nu), mu));
      fquat c = f_ld(L(h, par, id, nu));
      A = f_add(A, f_mul_bd(f_mul_bd(a, b), c));
    }
    if (!drop_bwd) {
      int m = id + minus(n, nu);
      fquat a = f_ld(L(h, par, m + plus(n, mu), nu));
      fquat b = f_ld(L(h, o, m, mu));
      fquat c = f_ld(L(h, o, m, nu));
      A = f_add(A, f_mul(f_mul_adbd(a, b), c));
    }
  }
  return A;
}

/* Kennedy-Pendleton (mc_updates.h:43-64) in float; the accept test in double
 * (1 - lf is within an ulp of 1 for a large coupling); the length of the
 * spatial part as n = 2 sqrt(lf (1 - lf)), free of cancellation */
static fquat heat_bath32(fquat A, float beta, pstream* st, int* tries_out) {
  float det = f_det(A), rinv = 1.0f / sqrtf(det), a = det * rinv;
  A = f_scale(A, rinv);
  float inv = 0.5f / (a * beta), lf = 0.f, aux;
  int tries = 0;
  for (tries = 1; tries <= 4096; tries++) {
    float r0 = ps_uniform(st), r1 = ps_uniform(st), r2 = ps_uniform(st);
    float c = -cosf(6.2831853f * (r1 - 0.5f));
    lf = -(logf(r0) + c * c * logf(r2)) * inv;
    aux = 1.f - ps_uniform(st);
    if (!((double)aux * aux > 1.0 - (double)lf)) break;
  }
  *tries_out = tries;
  float x0 = 1.f - 2.f * lf;
  float nrm = 2.f * sqrtf(lf * (1.f - lf));
  float ct = 2.f * ps_uniform(st) - 1.f;
  float ang = 6.2831853f * (ps_uniform(st) - 0.5f);
  float sp = sinf(ang), cp = cosf(ang);
  float stt = sqrtf(fmaxf(0.f, 1.f - ct * ct));
  fquat X = {x0, nrm * ct, -nrm * stt * cp, -nrm * stt * sp};
  return f_mul_bd(X, A);
}

/* mc_updates.h:16-36 in float, the action change and the accept test
 * (mc_updates.h:7-15) in double */
static int metropolis32(fquat* U, fquat A, float beta, float eps, int upd, pstream* st) {
  int acc = 0;
  const float r0 = sqrtf(1.f - eps * eps);
  for (int hit = 0; hit < upd; hit++) {
    float r1 = ps_uniform(st) - 0.5f, r2 = ps_uniform(st) - 0.5f, r3 = ps_uniform(st) - 0.5f;
    float sc = eps * (1.0f / sqrtf(r1 * r1 + r2 * r2 + r3 * r3));
    fquat r = {r0, sc * r1, sc * r2, sc * r3};
    fquat Un = f_mul(r, *U);
    fquat dU = {Un.w - U->w, Un.x - U->x, Un.y - U->y, Un.z - U->z};
    float retr = dU.w * A.w - dU.x * A.x - dU.y * A.y - dU.z * A.z;
    double s = -(double)beta * (double)retr;
    int ok = s < 0 ? 1 : metropolis_accept(s, ps_uniform_double(st));
    if (ok) {
      *U = Un;
      acc++;
    }
  }
  return acc;
}

/* mc_updates.h:109-115 in float, in the library's form: U' = 2 (<A, Ubar> /
 * |A|^2) Abar - U, which is (Ahat U Ahat)^+ by the quaternion identity
 * q p q = 2 <q, pbar> q - |q|^2 pbar */
static fquat over_relaxation32(fquat A, fquat U) {
  const float c = 2.f * (A.w * U.w - A.x * U.x - A.y * U.y - A.z * U.z) / f_det(A);
  return (fquat){c * A.w - U.w, -c * A.x - U.x, -c * A.y - U.y, -c * A.z - U.z};
}

/* re-projection with the norm taken in double */
static fquat renorm32(fquat u) {
  double d = (double)u.w * u.w + (double)u.x * u.x + (double)u.y * u.y + (double)u.z * u.z;
  double inv = 1.0 / sqrt(d);
  return (fquat){(float)(u.w * inv), (float)(u.x * inv), (float)(u.y * inv), (float)(u.z * inv)};
}

int ora_phase32(ora_lattice* h, int k, int kind, unsigned long long key, unsigned long long phase, int renorm,
                int* hb_tries) {
  if (!h || k < 0 || k > 5 || kind < 0 || kind > 2) return ORA_ERR_INVALID;
  const int mu = k / 2, par = k % 2;
  const float beta = h->p.beta;
#pragma omp parallel for schedule(static)
  for (int id = 0; id < h->vh; id++) {
    nbr_t n = nbr(h, id, par);
    if (h->p.boundary == 1 && mu != 0 && n.yq == 0 && n.q == 0) continue;
    fquat A = staples32(h, mu, par, id, &n);
    double* u = L(h, par, id, mu);
    size_t site = (size_t)par * h->vh + id;
    fquat U;
    if (kind == 1) {
      pstream st;
      ps_init(&st, key, (uint32_t)id, phase);
      int tries = 0;
      U = heat_bath32(A, beta, &st, &tries);
      if (hb_tries) hb_tries[site] = tries;
      h->accept[site] += 1;
    } else if (kind == 0) {
      pstream st;
      ps_init(&st, key, (uint32_t)id, phase);
      U = f_ld(u);
      h->accept[site] += metropolis32(&U, A, beta, h->p.epsilon, h->p.upd, &st);
    } else {
      U = over_relaxation32(A, f_ld(u));
      h->accept[site] += 1;
    }
    f_st(u, renorm ? renorm32(U) : U);
  }
  return h->err;
}

void ora_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) { philox4x32_10(ctr, key, out); }
