/*
 * pim_oracle.c - CPU restatement of the reference CPU_PIM hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker; see pim_oracle.h).  Line citations are to
 * CPU-PIM/CPU_PIM.cpp in the reference repository.
 */
#include "pim_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- random words */

/* Philox4x32-10 as published by Salmon et al. (SC'11): ten rounds of two 32x32->64
   multiplies, with the Weyl key schedule between rounds. */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

uint32_t orc_sweep_word(uint64_t seed, uint32_t group, uint32_t replica, uint32_t sweep,
                        uint32_t loc, int k) {
    uint32_t ctr[4] = {loc, sweep, replica, group};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t out[4];
    orc_philox4x32_10(ctr, key, out);
    return out[k & 3];
}

uint32_t orc_shuffle_word(uint64_t seed, uint64_t k) {
    uint32_t ctr[4] = {(uint32_t)(k >> 2), (uint32_t)(k >> 34), 0u, 0xFFFFFFFFu};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t out[4];
    orc_philox4x32_10(ctr, key, out);
    return out[k & 3];
}

/* std::generate_canonical<double, 53> over a 32-bit engine (CPU_PIM.cpp:212): two words,
   sum = w0 + w1 * 2^32 rounded once to double, divided by 2^64, clamped below 1. */
double orc_canonical(uint32_t w0, uint32_t w1) {
    double sum = (double)w0;
    sum += (double)w1 * 4294967296.0;
    double r = sum / 18446744073709551616.0;
    if (r >= 1.0) r = nextafter(1.0, 0.0);
    return r;
}

/* std::uniform_int_distribution<uint32>(0, range-1) over a 32-bit engine: Lemire's
   nearly-divisionless method ("Fast Random Integer Generation in an Interval", ACM TOMACS
   29(1), 2019), the algorithm the C++ library applies for a 32-bit engine. */
uint32_t orc_uniform_below(uint64_t seed, uint64_t *k, uint32_t range) {
    uint64_t product = (uint64_t)orc_shuffle_word(seed, (*k)++) * range;
    uint32_t low = (uint32_t)product;
    if (low < range) {
        uint32_t threshold = (uint32_t)(0u - range) % range;
        while (low < threshold) {
            product = (uint64_t)orc_shuffle_word(seed, (*k)++) * range;
            low = (uint32_t)product;
        }
    }
    return (uint32_t)(product >> 32);
}

/* ---------------------------------------------------------------- setup */

/* CPU_PIM.cpp:134-162: identity, then for each group t and location i one draw j from the
   shared stream (rng[0] in the reference) and the transposition (i j) for every replica. */
void orc_initial_perms(int n, int T, uint64_t seed, int32_t *phi) {
    uint64_t k = 0;
    for (int t = 0; t < T; ++t) {
        int32_t *p = phi + (size_t)t * n;
        for (int i = 0; i < n; ++i) p[i] = i;
        for (int i = 0; i < n; ++i) {
            int j = (int)orc_uniform_below(seed, &k, (uint32_t)n);
            if (i != j) {
                int32_t tmp = p[i];
                p[i] = p[j];
                p[j] = tmp;
            }
        }
    }
}

/* CPU_PIM.cpp:113-118: the last slot holds beta0, each lower slot is divided by deltaBeta. */
void orc_beta_ladder(int R, double beta0, double delta_beta, double *beta) {
    double running = beta0;
    for (int l = R - 1; l >= 0; --l) {
        beta[l] = running;
        running /= delta_beta;
    }
}

/* CPU_PIM.cpp:164-192:
     I[i][a] = -sum_j (D[i][j] F[a][phi(j)] + D[j][i] F[phi(j)][a])
     E       =  sum_ij D[i][j] F[phi(i)][phi(j)] */
void orc_force_init(int n, const int32_t *D, const int32_t *F, const int32_t *phi,
                    int64_t *I, int64_t *E) {
    for (int i = 0; i < n; ++i) {
        for (int a = 0; a < n; ++a) {
            int64_t acc = 0;
            for (int j = 0; j < n; ++j) {
                acc -= (int64_t)D[i * n + j] * F[a * n + phi[j]];
                acc -= (int64_t)D[j * n + i] * F[phi[j] * n + a];
            }
            I[(size_t)i * n + a] = acc;
        }
    }
    int64_t e = 0;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) e += (int64_t)D[i * n + j] * F[phi[i] * n + phi[j]];
    *E = e;
}

/* ---------------------------------------------------------------- the sweep */

/* (int)x of the reference (CPU_PIM.cpp:235): truncation toward zero; a value outside the
   integer range yields the most negative integer, as the x86 conversion instruction does. */
static int64_t trunc_cutoff(double x) {
    if (!(x > -9223372036854775808.0) || !(x < 9223372036854775808.0))
        return INT64_MIN;
    return (int64_t)x;
}

int orc_update(int n, const int32_t *D, const int32_t *F, int64_t *I, int32_t *phi,
               int32_t *phiinv, int64_t *E, int64_t *bestE, double beta, int i,
               uint32_t w0, uint32_t w1, int64_t *dE_out) {
    return orc_update_r(n, D, F, I, phi, phiinv, E, bestE, beta, i,
                        orc_canonical(w0, w1), dE_out);   /* r, :212 */
}

int orc_update_r(int n, const int32_t *D, const int32_t *F, int64_t *I, int32_t *phi,
                 int32_t *phiinv, int64_t *E, int64_t *bestE, double beta, int i, double r,
                 int64_t *dE_out) {
    long double probs[256];
    int64_t dEs[256];
    int64_t maxDeltaE = 0;                              /* :208, starts at 0 */
    double probSum = 0.0;
    const int a = phi[i];                               /* :215 */
    const int64_t *Ii = I + (size_t)i * n;
    for (int b = 0; b < n; ++b) {                       /* :220-232 */
        int j = phiinv[b];
        const int64_t *Ij = I + (size_t)j * n;
        int64_t dd = (int64_t)D[i * n + i] + D[j * n + j] - D[i * n + j] - D[j * n + i];
        int64_t ff = (int64_t)F[a * n + a] + F[b * n + b] - F[a * n + b] - F[b * n + a];
        int64_t dE = Ii[b] + Ij[a] - Ii[a] - Ij[b] - dd * ff;
        dEs[b] = dE;
        if (dE > maxDeltaE) maxDeltaE = dE;
    }
    if (dE_out) memcpy(dE_out, dEs, sizeof(int64_t) * (size_t)n);
    const double low_cutoff_double = (double)maxDeltaE - 20.0 / beta;   /* :234 */
    const int64_t cut = trunc_cutoff(low_cutoff_double);                 /* :235 */
    for (int b = 0; b < n; ++b) {                        /* :236-245 */
        probs[b] = 0.0L;
        if (dEs[b] > cut) {
            long double expr = (long double)(beta * (double)dEs[b]);
            probs[b] = exp2l(expr);
            probSum = (double)((long double)probSum + probs[b]);
        }
    }
    const double scaledR = r * probSum;                  /* :247 */
    double cumulativeProb = 0.0;
    for (int b = 0; b < n; ++b) {                        /* :249-287 */
        cumulativeProb = (double)((long double)cumulativeProb + probs[b]);
        if (cumulativeProb >= scaledR) {
            if (b != a) {
                int j = phiinv[b];
                *E -= dEs[b];                            /* :256 */
                phi[i] = b;
                phiinv[b] = i;
                phi[j] = a;
                phiinv[a] = j;
                /* :263-269, I[k][c] += d1(k) (F[c][b] - F[c][a]) + d2(k) (F[b][c] - F[a][c]),
                   with the two flow differences taken once per swap (integers: same sums) */
                int64_t colf[256], rowf[256];
                for (int c = 0; c < n; ++c) {
                    colf[c] = (int64_t)F[c * n + b] - F[c * n + a];
                    rowf[c] = (int64_t)F[b * n + c] - F[a * n + c];
                }
                for (int k = 0; k < n; ++k) {
                    const int64_t d1 = (int64_t)D[k * n + j] - D[k * n + i];
                    const int64_t d2 = (int64_t)D[j * n + k] - D[i * n + k];
                    int64_t *Ik = I + (size_t)k * n;
                    for (int c = 0; c < n; ++c) Ik[c] += d1 * colf[c] + d2 * rowf[c];
                }
                if (*E < *bestE) *bestE = *E;            /* :271-272 */
            }
            return b;
        }
    }
    return -1;
}

uint32_t orc_lumped_word(uint64_t seed, uint32_t group, uint32_t replica, uint32_t sweep,
                         uint32_t loc, uint32_t k) {
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t out[4];
    if (k < 2) {
        const uint32_t ctr[4] = {loc, sweep, replica, group};
        orc_philox4x32_10(ctr, key, out);
        return out[2 + k];
    }
    const uint32_t m = (k - 2) / 4 + 1;
    const uint32_t ctr[4] = {loc, sweep, replica, group + 0x10000u * m};
    orc_philox4x32_10(ctr, key, out);
    return out[(k - 2) % 4];
}

int orc_update_clique(int n, int act, const int32_t *D, const int32_t *F, int64_t *I,
                      int32_t *phi, int32_t *phiinv, int64_t *E, int64_t *bestE, double beta,
                      int i, uint32_t w0, uint32_t w1, uint64_t seed, uint32_t group,
                      uint32_t replica, uint32_t sweep) {
    long double probs[256];
    int64_t dEs[256];
    int64_t maxDeltaE = 0;
    const double r = orc_canonical(w0, w1);             /* :228 */
    double probSum = 0.0;
    const int a = phi[i];
    const int ncand = a < act ? n : act + 1;            /* :236, act = the lumped candidate */
    const int64_t *Ii = I + (size_t)i * n;
    for (int b = 0; b < ncand; ++b) {                   /* :236-249, zero diagonals */
        int j = phiinv[b];
        const int64_t *Ij = I + (size_t)j * n;
        int64_t dE = Ii[b] + Ij[a] - Ii[a] - Ij[b] -
                     (-(int64_t)D[i * n + j] - D[j * n + i]) * (-(int64_t)F[a * n + b] - F[b * n + a]);
        dEs[b] = dE;
        if (dE > maxDeltaE) maxDeltaE = dE;
    }
    const int64_t cut = trunc_cutoff((double)maxDeltaE - 20.0 / beta);   /* :251-252 */
    for (int b = 0; b < ncand; ++b) {                   /* :253-266 */
        probs[b] = 0.0L;
        const int lumped = a >= act && b == act;
        if (dEs[b] > cut || lumped) {
            long double expr = (long double)(beta * (double)dEs[b]);
            probs[b] = exp2l(expr);
            if (lumped) probs[b] *= (long double)(n - act);
            probSum = (double)((long double)probSum + probs[b]);
        }
    }
    const double scaledR = r * probSum;                  /* :268 */
    double cumulativeProb = 0.0;
    const int npick = a < act ? n : act;                 /* the lumped candidate is not scanned */
    for (int b = 0; b < npick; ++b) {                    /* :270-320 */
        cumulativeProb = (double)((long double)cumulativeProb + probs[b]);
        if (cumulativeProb >= scaledR) {
            if (b != a) {
                int j = phiinv[b];
                *E -= dEs[b];
                phi[i] = b;
                phiinv[b] = i;
                phi[j] = a;
                phiinv[a] = j;
                /* the reference's region-split update equals the full rank-2 update for a
                   clique of unit flows (:286-302) */
                for (int k = 0; k < n; ++k) {
                    int64_t d1 = (int64_t)D[k * n + j] - D[k * n + i];
                    int64_t d2 = (int64_t)D[j * n + k] - D[i * n + k];
                    int64_t *Ik = I + (size_t)k * n;
                    for (int c = 0; c < n; ++c)
                        Ik[c] += d1 * ((int64_t)F[c * n + b] - F[c * n + a]) +
                                 d2 * ((int64_t)F[b * n + c] - F[a * n + c]);
                }
                if (*E < *bestE) *bestE = *E;
            }
            return b;
        }
    }
    if (a >= act) {                                      /* :323-336, inactive to inactive */
        const uint32_t range = (uint32_t)(n - act);
        uint32_t k = 0;
        uint64_t product = (uint64_t)orc_lumped_word(seed, group, replica, sweep, (uint32_t)i, k++) * range;
        uint32_t low = (uint32_t)product;
        if (low < range) {
            uint32_t threshold = (uint32_t)(0u - range) % range;
            while (low < threshold) {
                product = (uint64_t)orc_lumped_word(seed, group, replica, sweep, (uint32_t)i, k++) * range;
                low = (uint32_t)product;
            }
        }
        const int b = act + (int)(product >> 32);
        const int j = phiinv[b];
        phi[i] = b;
        phiinv[b] = i;
        phi[j] = a;
        phiinv[a] = j;
        return b;
    }
    return -1;
}

int64_t orc_replica_sweeps(int n, const int32_t *D, const int32_t *F, int64_t *I,
                           int32_t *phi, int32_t *phiinv, int64_t *E, int64_t *bestE,
                           double beta, uint64_t seed, uint32_t group, uint32_t replica,
                           uint32_t sweep0, int nsweeps, int32_t *picks) {
    int64_t accepts = 0;
    for (int s = 0; s < nsweeps; ++s) {                  /* :206 */
        for (int i = 0; i < n; ++i) {                    /* :207 */
            uint32_t sw = sweep0 + (uint32_t)s;
            uint32_t w0 = orc_sweep_word(seed, group, replica, sw, (uint32_t)i, 0);
            uint32_t w1 = orc_sweep_word(seed, group, replica, sw, (uint32_t)i, 1);
            int a = phi[i];
            int b = orc_update(n, D, F, I, phi, phiinv, E, bestE, beta, i, w0, w1, 0);
            if (b >= 0 && b != a) ++accepts;
            if (picks) picks[(size_t)s * n + i] = b;
        }
    }
    return accepts;
}

int64_t orc_replay_sweeps(int n, const int32_t *D, const int32_t *F, int64_t *I, int32_t *phi,
                          int32_t *phiinv, int64_t *E, int64_t *bestE, double beta, int nsweeps,
                          const double *r, int32_t *picks) {
    int64_t accepts = 0;
    for (int s = 0; s < nsweeps; ++s) {
        for (int i = 0; i < n; ++i) {
            const int a = phi[i];
            const int b = orc_update_r(n, D, F, I, phi, phiinv, E, bestE, beta, i,
                                       r[(size_t)s * n + i], 0);
            if (b >= 0 && b != a) ++accepts;
            if (picks) picks[(size_t)s * n + i] = b;
        }
    }
    return accepts;
}

/* ---------------------------------------------------------------- one-shot parallel update */

/* 2^x in binary32 for x <= 0 (Cody-Waite reduction x = k + f, |f| <= 1/2, then the degree-7
   Taylor polynomial of 2^f = e^(f ln 2) by Horner's rule with fused multiply-adds, scaled by
   2^k).  Every step is one correctly rounded IEEE operation, so the solver's device copy of
   this function returns the same bits.  Error below 1 ulp over the normal range. */
static const float kExp2Coef[8] = {0x1p+0f,         0x1.62e430p-1f, 0x1.ebfbe0p-3f,
                                   0x1.c6b08ep-5f,  0x1.3b2ab6p-7f, 0x1.5d87fep-10f,
                                   0x1.430912p-13f, 0x1.ffcbfcp-17f};

static float bits_float(uint32_t u) {
    float f;
    memcpy(&f, &u, 4);
    return f;
}

float orc_exp2f_neg(float x) {
    if (!(x > -150.0f)) return 0.0f;
    if (x > 0.0f) x = 0.0f;
    const float k = rintf(x);
    const float f = x - k;                               /* exact */
    float p = kExp2Coef[7];
    for (int c = 6; c >= 0; --c) p = fmaf(p, f, kExp2Coef[c]);
    const int ki = (int)k;
    if (ki >= -126) return p * bits_float((uint32_t)(ki + 127) << 23);
    return (p * bits_float((uint32_t)(ki + 64 + 127) << 23)) * 0x1p-64f;
}

/* The threshold of a one-shot proposal: word 0 of the update's Philox block as an odd
   multiple of 2^-24, in (0, 1). */
float orc_oneshot_uniform(uint32_t w0) {
    return (float)(((w0 >> 9) << 1) | 1u) * 0x1p-24f;
}

void orc_oneshot_uniforms(uint64_t seed, int count, int R, uint32_t step, int n, float *out) {
    for (int k = 0; k < count; ++k)
        for (int i = 0; i < n; ++i)
            out[(size_t)k * n + i] = orc_oneshot_uniform(
                orc_sweep_word(seed, (uint32_t)(k / R), (uint32_t)(k % R), step, (uint32_t)i, 0));
}

/* The proposal of one location (GPU-CUPIM qap.cu:1040-1146, os_pwc_d): deltas d[j] of every
   partner location j, weights 2^(beta (d[j] - max)) in binary32 with no cutoff, summed in the
   reference's warp order (lane t holds j = t, t+32, ...: a running sum per lane, then an
   inclusive Hillis-Steele scan of the lane totals over 32 lanes), and the first lane whose
   span [prev, cur) contains u * total picks its j; when no lane does, j = n - 1
   (:1136-1144).  Returns j; *delta_out = d[j]. */
int orc_oneshot_pick(int n, const int64_t *d, float beta_f, float u, int64_t *delta_out) {
    int64_t mx = d[0];
    for (int j = 1; j < n; ++j)
        if (d[j] > mx) mx = d[j];
    const int K = (n + 31) / 32;
    float s[32][8], tot[32], x[32], y[32], off[32];
    for (int t = 0; t < 32; ++t) {
        float run = 0.0f;
        for (int k = 0; k < K; ++k) {
            const int j = t + 32 * k;
            const float w = (j < n) ? orc_exp2f_neg(beta_f * (float)(d[j] - mx)) : 0.0f;
            run = (k == 0) ? w : w + run;                /* :1094-1099 */
            s[t][k] = run;
        }
        tot[t] = run;
        x[t] = run;
    }
    for (int dd = 1; dd < 32; dd <<= 1) {                /* :1101-1110 */
        for (int t = 0; t < 32; ++t) y[t] = (t >= dd) ? x[t] + x[t - dd] : x[t];
        memcpy(x, y, sizeof(x));
    }
    for (int t = 0; t < 32; ++t) off[t] = x[t] - tot[t];
    const float total = off[31] + tot[31];
    const float thresh = u * total;                      /* :1114 */
    for (int t = 0; t < 32; ++t) {                       /* :1119-1135, lowest lane wins */
        int win = -1;
        for (int k = 0; k < K; ++k) {
            const int j = t + 32 * k;
            if (j >= n) break;
            const float cur = off[t] + s[t][k];
            const float prev = (k == 0) ? off[t] : off[t] + s[t][k - 1];
            if (cur >= thresh && prev < thresh) win = j;
        }
        if (win >= 0) {
            *delta_out = d[win];
            return win;
        }
    }
    *delta_out = d[n - 1];
    return n - 1;
}

/* Ballot word of a proposal (i -> target with delta): the larger delta wins, then the lower i
   (GPU-CUPIM qap.cu:1184-1198); deltas beyond int32 are saturated (the reference's are int32). */
static uint64_t oneshot_ballot(int64_t delta, int i) {
    const int32_t d32 = delta > INT32_MAX ? INT32_MAX : (delta < INT32_MIN ? INT32_MIN : (int32_t)delta);
    const uint32_t biased = ~((uint32_t)d32 ^ 0x80000000u);
    return ((uint64_t)biased << 32) | (uint32_t)i;
}

int orc_oneshot_step(int n, const int32_t *D, const int32_t *F, int64_t *I, int32_t *phi,
                     int32_t *phiinv, int64_t *E, int64_t *bestE, double beta, uint64_t seed,
                     uint32_t group, uint32_t replica, uint32_t step, int32_t *targets) {
    int32_t tgt[256], acc_i[256], acc_j[256], acc_a[256], acc_b[256];
    int64_t dl[256], d[256];
    uint64_t own[256];
    const float beta_f = (float)beta;
    /* 1. every location proposes against the same snapshot */
    for (int i = 0; i < n; ++i) {
        const int a = phi[i];
        const int64_t *Ii = I + (size_t)i * n;
        for (int j = 0; j < n; ++j) {                    /* qap.cu:609-646 */
            const int b = phi[j];
            const int64_t dd = (int64_t)D[i * n + i] + D[j * n + j] - D[i * n + j] - D[j * n + i];
            const int64_t ff = (int64_t)F[a * n + a] + F[b * n + b] - F[a * n + b] - F[b * n + a];
            d[j] = Ii[b] + I[(size_t)j * n + a] - Ii[a] - I[(size_t)j * n + b] - dd * ff;
        }
        const float u = orc_oneshot_uniform(orc_sweep_word(seed, group, replica, step, (uint32_t)i, 0));
        tgt[i] = orc_oneshot_pick(n, d, beta_f, u, &dl[i]);
        if (targets) targets[i] = tgt[i];
    }
    /* 2. collisions: a location goes to the best ballot touching it (qap.cu:1150-1225) */
    for (int i = 0; i < n; ++i) own[i] = UINT64_MAX;
    for (int i = 0; i < n; ++i) {
        if (tgt[i] == i) continue;
        const uint64_t w = oneshot_ballot(dl[i], i);
        if (w < own[tgt[i]]) own[tgt[i]] = w;
        if (w < own[i]) own[i] = w;
    }
    int np = 0;
    for (int i = 0; i < n; ++i) {
        const int j = tgt[i];
        if (j == i || (uint32_t)own[i] != (uint32_t)i || (uint32_t)own[j] != (uint32_t)i) continue;
        acc_i[np] = i;
        acc_j[np] = j;
        acc_a[np] = phi[i];
        acc_b[np] = phi[j];
        ++np;
    }
    /* 3. the accepted swaps are disjoint, so their rank-2 force updates add up exactly
          (qap.cu:1337-1412); facilities are those before the step */
    for (int p = 0; p < np; ++p) {
        const int i = acc_i[p], j = acc_j[p], a = acc_a[p], b = acc_b[p];
        for (int k = 0; k < n; ++k) {
            const int64_t u1 = (int64_t)D[k * n + j] - D[k * n + i];
            const int64_t u2 = (int64_t)D[j * n + k] - D[i * n + k];
            int64_t *Ik = I + (size_t)k * n;
            for (int c = 0; c < n; ++c)
                Ik[c] += u1 * ((int64_t)F[c * n + b] - F[c * n + a]) +
                         u2 * ((int64_t)F[b * n + c] - F[a * n + c]);
        }
    }
    for (int p = 0; p < np; ++p) {                       /* qap.cu:1311-1332 */
        const int i = acc_i[p], j = acc_j[p], a = acc_a[p], b = acc_b[p];
        phi[i] = b;
        phi[j] = a;
        phiinv[a] = j;
        phiinv[b] = i;
    }
    /* 4. the energy from the new force matrix, E = -1/2 sum_k I[k][phi(k)] (qap.cu:1420-1458) */
    int64_t sum = 0;
    for (int k = 0; k < n; ++k) sum += I[(size_t)k * n + phi[k]];
    *E = -sum / 2;
    if (*E < *bestE) *bestE = *E;
    return np;
}

/* ---------------------------------------------------------------- tracking + exchange */

int orc_track_exchange(int R, int cap, const int64_t *E, const int64_t *bestE, double *beta,
                       int32_t *order, int32_t *time_since_swap, int64_t *thread_best,
                       int64_t *single_best) {
    int found_better = 0;
    (*time_since_swap)++;                                /* :295 */
    for (int l = 0; l < R; ++l) {                        /* :297-314 */
        if (bestE[l] < *thread_best) {
            found_better = 1;
            *thread_best = bestE[l];
            *time_since_swap = 0;
            if (*thread_best < *single_best) *single_best = *thread_best;
        }
    }
    for (int l = 0; l < R - 1; ++l) {                    /* :324-337, coldest rank last */
        int i1 = order[l], i2 = order[l + 1];
        double e1 = (double)E[i1], e2 = (double)E[i2];
        if (e1 < e2) {
            order[l] = i2;
            order[l + 1] = i1;
            double tb = beta[i1];
            beta[i1] = beta[i2];
            beta[i2] = tb;
            if (i2 == R - 1) *time_since_swap = 0;       /* compares a replica index (:333) */
        }
    }
    if (*time_since_swap > 100) {                        /* :339-344, slot cap-1 */
        int i1 = order[cap - 1], i2 = order[0];
        order[cap - 1] = i2;
        order[0] = i1;
        double tb = beta[i1];
        beta[i1] = beta[i2];
        beta[i2] = tb;
    }
    return found_better;
}

/* ---------------------------------------------------------------- whole run */

void orc_setup(orc_run_state *st, const int32_t *D, const int32_t *F, double beta0,
               double delta_beta) {
    const int n = st->n, T = st->T, R = st->R;
    for (int t = 0; t < T; ++t) {
        st->time_since_swap[t] = 0;
        st->thread_best[t] = ORC_NO_BEST;
        orc_beta_ladder(R, beta0, delta_beta, st->beta + (size_t)t * R);
        for (int l = 0; l < st->cap; ++l) st->order[(size_t)t * st->cap + l] = (l < R) ? l : 0;
    }
    st->single_best = ORC_NO_BEST;
    st->megaiters_done = 0;
    st->accepts = 0;
    st->target_megaiter = -1;
    /* one shuffle stream for all groups, drawn group after group (CPU_PIM.cpp:145-148) */
    int32_t *perms = (int32_t *)malloc(sizeof(int32_t) * (size_t)T * n);
    orc_initial_perms(n, T, st->seed, perms);
    for (int t = 0; t < T; ++t) {
        for (int l = 0; l < R; ++l) {
            size_t rep = (size_t)t * R + l;
            int32_t *phi = st->phi + rep * n;
            int32_t *inv = st->phiinv + rep * n;
            memcpy(phi, perms + (size_t)t * n, sizeof(int32_t) * (size_t)n);
            for (int i = 0; i < n; ++i) inv[phi[i]] = i;
            st->bestE[rep] = ORC_NO_BEST;
            orc_force_init(n, D, F, phi, st->I + rep * (size_t)n * n, &st->E[rep]);
        }
    }
    free(perms);
}

int orc_run(orc_run_state *st, const int32_t *D, const int32_t *F, int64_t megaiters,
            int64_t goal) {
    const int n = st->n, T = st->T, R = st->R;
    for (int64_t m = 0; m < megaiters; ++m) {
        for (int t = 0; t < T; ++t) {
            size_t r0 = (size_t)t * R;
            orc_track_exchange(R, st->cap, st->E + r0, st->bestE + r0, st->beta + r0,
                               st->order + (size_t)t * st->cap, &st->time_since_swap[t],
                               &st->thread_best[t], &st->single_best);
        }
        if (st->single_best <= goal) {                   /* :346-348 */
            if (st->target_megaiter < 0) st->target_megaiter = st->megaiters_done;
            return 1;
        }
        uint32_t sweep0 = (uint32_t)(st->megaiters_done * st->numitera);
        /* :360-362.  The replicas' sweeps between two exchanges touch only their own state,
           so they run in parallel (the reference runs its groups on threads too); the
           results do not depend on the schedule. */
        int64_t acc = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : acc)
        for (int q = 0; q < T * R; ++q) {
            {
                const int t = q / R, l = q % R;
                size_t rep = (size_t)q;
                if (st->rule == 1) {
                    for (int s2 = 0; s2 < st->numitera; ++s2)
                        acc += orc_oneshot_step(
                            n, D, F, st->I + rep * (size_t)n * n, st->phi + rep * n, st->phiinv + rep * n,
                            &st->E[rep], &st->bestE[rep], st->beta[rep], st->seed, (uint32_t)t,
                            (uint32_t)l, sweep0 + (uint32_t)s2, 0);
                    continue;
                }
                if (st->active > 0) {
                    for (int s2 = 0; s2 < st->numitera; ++s2)
                        for (int i = 0; i < n; ++i) {
                            const uint32_t sw = sweep0 + (uint32_t)s2;
                            const int a = st->phi[rep * n + i];
                            const int b = orc_update_clique(
                                n, st->active, D, F, st->I + rep * (size_t)n * n, st->phi + rep * n,
                                st->phiinv + rep * n, &st->E[rep], &st->bestE[rep], st->beta[rep], i,
                                orc_sweep_word(st->seed, (uint32_t)t, (uint32_t)l, sw, (uint32_t)i, 0),
                                orc_sweep_word(st->seed, (uint32_t)t, (uint32_t)l, sw, (uint32_t)i, 1),
                                st->seed, (uint32_t)t, (uint32_t)l, sw);
                            if (b >= 0 && b != a) acc++;
                        }
                    continue;
                }
                acc += orc_replica_sweeps(
                    n, D, F, st->I + rep * (size_t)n * n, st->phi + rep * n,
                    st->phiinv + rep * n, &st->E[rep], &st->bestE[rep], st->beta[rep],
                    st->seed, (uint32_t)t, (uint32_t)l, sweep0, st->numitera, 0);
            }
        }
        st->accepts += acc;
        st->megaiters_done++;
    }
    return 0;
}
