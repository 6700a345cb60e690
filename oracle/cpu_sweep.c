/*
 * cpu_sweep.c — the colour-class sweep restated in C for the host cores (ORACLE: test infrastructure and the
 * timed CPU baseline only; never linked into the product).
 *
 * Same arithmetic as the reference's generated class kernel (Spin_Colour_Kernel/generator.py:150-319) in
 * float32 with no FMA contraction (built with -ffp-contract=off): local field by coupling groups, extra
 * matrices and field; Philox4x32-10 proposals keyed per sweep; cubic anisotropy; Metropolis or Barker. The
 * reference's CPU path evaluates exp with NumPy's float32 exp, which differs from the C library's expf in the
 * last bits for a large share of arguments; Ising energy changes form a finite set, so for Ising the caller
 * passes, per replica, the sorted arguments the chain can reach with NumPy's exp of each, and the port looks
 * the exact argument up (bit-exact Ising chains). Vector models take cos, sin, exp and sqrt from the C library
 * and agree with the NumPy oracle within float32 rounding, not bit for bit. Replicas run in parallel over
 * OpenMP threads; each replica's sites are visited class by class, which equals the parallel class update
 * because no bond joins two sites of a class.
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

/* exp of an Ising argument from the caller's table: xs[0..n) sorted ascending, es the matching values; sets *miss
 * when the argument is absent (the caller's enumeration did not cover it). */
typedef struct {
  const float* xs;
  const float* es;
  int64_t n;
} or_exp_table;

static float table_exp(const or_exp_table* t, float x, int* miss) {
  int64_t lo = 0, hi = t->n - 1;
  while (lo <= hi) {
    const int64_t mid = (lo + hi) / 2;
    const float v = t->xs[mid];
    if (v == x) return t->es[mid];
    if (v < x) lo = mid + 1; else hi = mid - 1;
  }
  *miss = 1;
  return expf(x);
}

static void site_update(const or_desc* d, float* S, const float* k1, const int8_t* mask, int64_t rep, float beta,
                        int alpha, int x, int y, int z, uint32_t k0, uint32_t k1w, const or_exp_table* et,
                        int* miss) {
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
  if (d->acceptance == 1) {
    const float xa = beta * dE;
    acc = u0 * (1.0f + (et ? table_exp(et, xa, miss) : expf(xa))) < 1.0f;
  } else {
    const float xa = -beta * dE;
    acc = u0 < (et ? table_exp(et, xa, miss) : expf(xa));
  }
  if (acc)
    for (int k = 0; k < n; ++k) R[(size_t)k * nsite + own] = t[k];
}

/* n_sweeps sweeps of B replicas, S = [B][n][b][L3][L2][L1] float32; reps[i] = global replica index of row i.
 * Ising exp tables (may be NULL): replica row i's arguments are exp_x[exp_off[i] .. exp_off[i + 1]), sorted, with
 * NumPy's exp of each in exp_e. Returns 0, or 1 when an argument was missing from a table. */
int oracle_sweep(const or_desc* d, float* S, const float* beta, const float* k1, const int8_t* mask, int B,
                 const int64_t* reps, int64_t base_seed, int64_t sweep0, int n_sweeps, int threads,
                 const float* exp_x, const float* exp_e, const int64_t* exp_off) {
  const int L1 = d->L[0], L2 = d->L[1], L3 = d->L[2];
  const size_t nsite = (size_t)d->b * L1 * L2 * L3;
  int missed = 0;
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 1) reduction(| : missed)
  for (int i = 0; i < B; ++i) {
    float* R = S + (size_t)i * d->n * nsite;
    or_exp_table et = {0, 0, 0};
    if (exp_x) {
      et.xs = exp_x + exp_off[i];
      et.es = exp_e + exp_off[i];
      et.n = exp_off[i + 1] - exp_off[i];
    }
    int miss = 0;
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
                site_update(d, R, k1, mask, reps ? reps[i] : i, beta[i], alpha, x, y, z, k0, k1w,
                            exp_x ? &et : 0, &miss);
      }
    }
    missed |= miss;
  }
  return missed;
}

int oracle_max_threads(void) { return omp_get_max_threads(); }

/* ------------------------------------------------------------------------------------------- bitwise Ising
 * The reference's multi-spin-coded chain (Spin_Colour_Kernel/bitwise.py:59-246, restated in oracle/bitwise.py)
 * on unpacked int8 spins S[B][b][L3][L2][L1] (+-1, 0 on masked sites): word w holds replicas 32 w .. 32 w + 31;
 * for a class site with z_eff present neighbours (inside the box and the mask, bonds of applied couplings) and
 * k anti-aligned ones, replica r flips when its draw is below table[w][s][z_eff][k] (s = 1 for spin +1 when the
 * system has a field, else 0).
 *   shared:      one float32 uniform per (word, site, sweep): output w % 4 of Philox(int32((w / 4) nsite + site));
 *   independent: one 32-bit integer U per (replica, site, sweep), bit 31 - l of replica 32 w + j's U = bit j of
 *                R_l, R_{4g+q} = output q of Philox(int32(w nsite + site)) under key_g =
 *                (key + (g + 1) 104729) mod 2147483629 (floored); flip iff U < P (int64 table).
 * words[lw] = global word index of local word lw (its counters); table rows follow local words. Sites of one
 * class run in parallel over OpenMP threads (no bond joins two sites of a class). */
static int32_t sweep_key_of(int64_t base_seed, int64_t sweep) {
  uint64_t v = (uint64_t)base_seed * 1000003ull + (uint64_t)sweep * 7919ull + 12345ull;
  return (int32_t)((int64_t)v % 2147483629ll);
}

int oracle_bitwise_sweep(const or_desc* d, int8_t* S, const int8_t* mask, int B, const int64_t* words,
                         const void* table, int Z1, int has_field, int independent, int64_t base_seed,
                         int64_t sweep0, int n_sweeps, int threads) {
  const int L1 = d->L[0], L2 = d->L[1], L3 = d->L[2];
  const int plane = L1 * L2 * L3, nsite = d->b * plane;
  const int W = (B + 31) / 32;
  if (threads > 0) omp_set_num_threads(threads);
  for (int sw = 0; sw < n_sweeps; ++sw) {
    const int32_t key = sweep_key_of(base_seed, sweep0 + sw);
    const uint32_t k0 = (uint32_t)key, k1 = key < 0 ? 0xFFFFFFFFu : 0u;
    uint32_t kg[8];
    for (int g = 0; g < 8; ++g) {
      int64_t r = ((int64_t)key + (int64_t)(g + 1) * 104729) % 2147483629ll;
      kg[g] = (uint32_t)(r < 0 ? r + 2147483629ll : r);
    }
    for (int ci = 0; ci < d->n_classes; ++ci) {
      const int colour = d->classes[ci][0], a = d->classes[ci][1];
#pragma omp parallel for schedule(static)
      for (int rem = 0; rem < plane; ++rem) {
        const int x = rem % L1, y = (rem / L1) % L2, z = rem / (L1 * L2);
        const int site = a * plane + rem;
        if (colour_of(d, a, x, y, z) != colour || (mask && !mask[site])) continue;
        int q[OR_MAX_BONDS], nq = 0;
        int bi = 0;
        for (int g = 0; g < d->n_groups[a]; ++g) {
          for (; bi < d->group_end[a][g]; ++bi) {
            if (!d->apply[a][g]) continue;
            const or_bond* bd = &d->bonds[a][bi];
            const int qx = axis(x, bd->dx, L1, d->periodic[0]), qy = axis(y, bd->dy, L2, d->periodic[1]);
            const int qz = axis(z, bd->dz, L3, d->periodic[2]);
            if (qx < 0 || qy < 0 || qz < 0) continue;
            const int qs = bd->a2 * plane + (qz * L2 + qy) * L1 + qx;
            if (mask && !mask[qs]) continue;
            q[nq++] = qs;
          }
        }
        for (int lw = 0; lw < W; ++lw) {
          const int64_t gw = words ? words[lw] : lw;
          float u = 0.0f;
          uint32_t R[32];
          if (!independent) {
            uint32_t out[4];
            philox((uint32_t)((uint64_t)(gw / 4) * (uint64_t)nsite + (uint64_t)site), k0, k1, out);
            u = uniform(out[gw % 4]);
          } else {
            for (int g = 0; g < 8; ++g)
              philox((uint32_t)((uint64_t)gw * (uint64_t)nsite + (uint64_t)site), kg[g], 0u, &R[4 * g]);
          }
          for (int j = 0; j < 32; ++j) {
            const int r = 32 * lw + j;
            if (r >= B) break;
            int8_t* Rr = S + (size_t)r * nsite;
            const int s = Rr[site];
            int tot = 0;
            for (int i = 0; i < nq; ++i) tot += Rr[q[i]];
            const int kk = (nq - s * tot) / 2;
            const int sidx = has_field ? (s > 0) : 0;
            const size_t ti = (((size_t)lw * 2 + sidx) * Z1 + nq) * Z1 + kk;
            int flip;
            if (!independent) {
              flip = u < ((const float*)table)[ti];
            } else {
              uint64_t U = 0;
              for (int l = 0; l < 32; ++l) U |= (uint64_t)((R[l] >> j) & 1u) << (31 - l);
              flip = (int64_t)U < ((const int64_t*)table)[ti];
            }
            if (flip) Rr[site] = (int8_t)(-s);
          }
        }
      }
    }
  }
  return 0;
}
