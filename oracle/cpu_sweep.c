/*
 * cpu_sweep.c — the colour-class sweep restated in C for the host cores (ORACLE: test infrastructure and the
 * timed CPU baseline only; never linked into the product).
 *
 * Same arithmetic as the reference's generated class kernel (Spin_Colour_Kernel/generator.py:150-319) in
 * float32 with no FMA contraction (built with -ffp-contract=off): local field by coupling groups, extra
 * matrices and field; Philox4x32-10 proposals keyed per sweep; cubic anisotropy; Metropolis or Barker. cos,
 * sin, exp and sqrt come from the C library, so vector-model trajectories agree with the NumPy oracle within
 * float32 rounding, not bit for bit. Replicas run in parallel over OpenMP threads; each replica's sites are
 * visited class by class, which equals the parallel class update because no bond joins two sites of a class.
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <string.h>

#define OR_MAX_BASIS 4
#define OR_MAX_BONDS 64
#define OR_MAX_GROUPS 8
#define OR_MAX_EXTRA 8

typedef struct {
  int32_t a2, dx, dy, dz, extra;
} or_bond;

typedef struct {
  int32_t n, b, L[3], periodic[3], acceptance; /* acceptance: 0 Metropolis, 1 Barker */
  float h[3];
  int32_t has_cubic;
  float k2;
  int32_t r, m[4], K[4][3], o[OR_MAX_BASIS][4];
  int32_t n_classes, classes[128][2];
  int32_t n_bonds[OR_MAX_BASIS], n_groups[OR_MAX_BASIS], group_end[OR_MAX_BASIS][OR_MAX_GROUPS];
  float J[OR_MAX_BASIS][OR_MAX_GROUPS];
  int32_t apply[OR_MAX_BASIS][OR_MAX_GROUPS];
  int32_t n_extra[OR_MAX_BASIS];
  float E[OR_MAX_BASIS][OR_MAX_EXTRA][9];
  or_bond bonds[OR_MAX_BASIS][OR_MAX_BONDS];
} or_desc;

int oracle_desc_size(void) { return (int)sizeof(or_desc); }

static inline uint32_t mulhi32(uint32_t a, uint32_t b) { return (uint32_t)(((uint64_t)a * b) >> 32); }

/* Philox4x32-10, counter (c0, 0, 0, 0), key (k0, k1). */
static void philox(uint32_t c0, uint32_t k0, uint32_t k1, uint32_t out[4]) {
  uint32_t x0 = c0, x1 = 0, x2 = 0, x3 = 0;
  for (int i = 0; i < 10; ++i) {
    uint32_t la = 0xD2511F53u * x0, ha = mulhi32(0xD2511F53u, x0);
    uint32_t lb = 0xCD9E8D57u * x2, hb = mulhi32(0xCD9E8D57u, x2);
    x0 = hb ^ x1 ^ k0;
    x2 = ha ^ x3 ^ k1;
    x1 = lb;
    x3 = la;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = x0; out[1] = x1; out[2] = x2; out[3] = x3;
}

static inline float uniform(uint32_t bits) {
  int32_t i = (int32_t)bits;
  if (i < 0) i = ~i;
  return (float)i * 4.6566127342e-10f;
}

static int colour_of(const or_desc* d, int a, int x, int y, int z) {
  int idx = 0;
  for (int r = 0; r < d->r; ++r) idx = idx * d->m[r] + (d->K[r][0] * x + d->K[r][1] * y + d->K[r][2] * z + d->o[a][r]) % d->m[r];
  return idx;
}

static inline int axis(int x, int dx, int L, int per) {
  int q = x + dx;
  if (per) { q %= L; if (q < 0) q += L; return q; }
  return (q >= 0 && q < L) ? q : -1;
}

static void site_update(const or_desc* d, float* S, const float* k1, const int8_t* mask, int64_t rep, float beta,
                        int alpha, int x, int y, int z, uint32_t k0, uint32_t k1w) {
  const int n = d->n, L1 = d->L[0], L2 = d->L[1], L3 = d->L[2];
  const int plane = L1 * L2 * L3, nsite = d->b * plane;
  const int own = alpha * plane + (z * L2 + y) * L1 + x;
  if (mask && !mask[own]) return;
  float* R = S;   /* this replica's block: n planes of nsite */
  float s[3] = {0, 0, 0}, v[3] = {0, 0, 0}, ex[OR_MAX_EXTRA][3];
  for (int k = 0; k < n; ++k) s[k] = R[(size_t)k * nsite + own];
  int bi = 0;
  for (int g = 0; g < d->n_groups[alpha]; ++g) {
    float gs[3] = {0, 0, 0};
    for (; bi < d->group_end[alpha][g]; ++bi) {
      const or_bond* bd = &d->bonds[alpha][bi];
      int qx = axis(x, bd->dx, L1, d->periodic[0]), qy = axis(y, bd->dy, L2, d->periodic[1]);
      int qz = axis(z, bd->dz, L3, d->periodic[2]);
      int q = (qx < 0 || qy < 0 || qz < 0) ? -1 : bd->a2 * plane + (qz * L2 + qy) * L1 + qx;
      for (int k = 0; k < n; ++k) {
        float t = q >= 0 ? R[(size_t)k * nsite + q] : 0.0f;
        gs[k] = gs[k] + t;
        if (bd->extra >= 0) ex[bd->extra][k] = t;
      }
    }
    if (d->apply[alpha][g])
      for (int k = 0; k < n; ++k) v[k] = v[k] + d->J[alpha][g] * gs[k];
  }
  for (int e = 0; e < d->n_extra[alpha]; ++e)
    for (int k = 0; k < n; ++k) {
      float tot = 0.0f;
      int any = 0;
      for (int l = 0; l < n; ++l) {
        float c = d->E[alpha][e][3 * k + l];
        if (c != 0.0f) { float term = c * ex[e][l]; tot = any ? tot + term : term; any = 1; }
      }
      if (any) v[k] = v[k] + tot;
    }
  for (int k = 0; k < n; ++k)
    if (d->h[k] != 0.0f) v[k] = v[k] + d->h[k];
  uint32_t rnd[4];
  philox((uint32_t)((uint64_t)rep * (uint64_t)nsite + (uint64_t)own), k0, k1w, rnd);
  const float u0 = uniform(rnd[0]);
  float t[3] = {0, 0, 0};
  if (n == 1) {
    t[0] = -s[0];
  } else if (n == 2) {
    float phi = 6.2831855f * uniform(rnd[1]);
    t[0] = cosf(phi);
    t[1] = sinf(phi);
  } else {
    float cz = 2.0f * uniform(rnd[1]) - 1.0f;
    float phi = 6.2831855f * uniform(rnd[2]);
    float rr = sqrtf(fmaxf(1.0f - cz * cz, 0.0f));
    t[0] = rr * cosf(phi);
    t[1] = rr * sinf(phi);
    t[2] = cz;
  }
  float acc_sum = (t[0] - s[0]) * v[0];
  for (int k = 1; k < n; ++k) acc_sum = acc_sum + (t[k] - s[k]) * v[k];
  float dE = -acc_sum;
  if (n == 3 && d->has_cubic) {
    const float kk = k1[own];
    float at, as;
    {
      float q01 = t[0] * t[1], q02 = t[0] * t[2], q12 = t[1] * t[2], tri = q01 * t[2];
      at = kk * ((q01 * q01 + q02 * q02) + q12 * q12) + (d->k2 * tri) * tri;
    }
    {
      float q01 = s[0] * s[1], q02 = s[0] * s[2], q12 = s[1] * s[2], tri = q01 * s[2];
      as = kk * ((q01 * q01 + q02 * q02) + q12 * q12) + (d->k2 * tri) * tri;
    }
    dE = dE + (at - as);
  }
  int acc;
  if (d->acceptance == 1)
    acc = u0 * (1.0f + expf(beta * dE)) < 1.0f;
  else
    acc = u0 < expf(-beta * dE);
  if (acc)
    for (int k = 0; k < n; ++k) R[(size_t)k * nsite + own] = t[k];
}

/* n_sweeps sweeps of B replicas, S = [B][n][b][L3][L2][L1] float32; reps[i] = global replica index of row i. */
int oracle_sweep(const or_desc* d, float* S, const float* beta, const float* k1, const int8_t* mask, int B,
                 const int64_t* reps, int64_t base_seed, int64_t sweep0, int n_sweeps, int threads) {
  const int L1 = d->L[0], L2 = d->L[1], L3 = d->L[2];
  const size_t nsite = (size_t)d->b * L1 * L2 * L3;
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 1)
  for (int i = 0; i < B; ++i) {
    float* R = S + (size_t)i * d->n * nsite;
    for (int sw = 0; sw < n_sweeps; ++sw) {
      uint64_t v = (uint64_t)base_seed * 1000003ull + (uint64_t)(sweep0 + sw) * 7919ull + 12345ull;
      int32_t key = (int32_t)((int64_t)v % 2147483629ll);
      uint32_t k0 = (uint32_t)key, k1w = key < 0 ? 0xFFFFFFFFu : 0u;
      for (int ci = 0; ci < d->n_classes; ++ci) {
        const int colour = d->classes[ci][0], alpha = d->classes[ci][1];
        for (int z = 0; z < L3; ++z)
          for (int y = 0; y < L2; ++y)
            for (int x = 0; x < L1; ++x)
              if (colour_of(d, alpha, x, y, z) == colour)
                site_update(d, R, k1, mask, reps ? reps[i] : i, beta[i], alpha, x, y, z, k0, k1w);
      }
    }
  }
  return 0;
}

int oracle_max_threads(void) { return omp_get_max_threads(); }
