/*
 * oracle/transport.c — TEST INFRASTRUCTURE, not part of the product.
 *
 * A CPU restatement of pyRadMC's coupled photon-electron transport, used only
 * by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg as the
 * checker and the timed CPU baseline.  Nothing in pyradmc_b200/ links or calls
 * it.  It follows the reference's own one-history-at-a-time oracle:
 *
 *   transport_history      pyradmc/transport/history.py:31-150 (LIFO stack)
 *   photon_steps           pyradmc/transport/photon.py:100-282
 *   electron_steps         pyradmc/transport/electron.py:207-481
 *   samplers               pyradmc/physics/{path,channel,compton,direction,
 *                          roulette,brems,moller,msc,gs,rayleigh}.py
 *   geometry               pyradmc/geometry/grid.py:35-223
 *   table lookups          pyradmc/data/tables.py:83-133 (float64 tables)
 *   batch statistics       pyradmc/scoring/dij.py:155-191, dose.py:169-207
 *
 * Arithmetic is float64 throughout, on the float64 flattened tables (the
 * reference engine queries its source directly; the tables reproduce those
 * queries to the 2e-4 parity budget of data/tables.py:56-58).  Scoring is int64
 * fixed point in 1e-9 MeV quanta with atomic adds (pthreads share the histories
 * of a batch), so the result does not depend on the thread count.  Random numbers come from Philox4x32-10 (Salmon et al.,
 * SC'11) keyed on (seed, history key), one sequential stream per history as in
 * the reference's HostRNG (rng/host.py:36-44); they are not the reference's
 * PCG64 streams, so agreement with pyRadMC is statistical, never bitwise.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <pthread.h>
#include <unistd.h>

#define ME 0.51099895069
#define ROULETTE_MEV 0.5
#define ROULETTE_SURVIVAL 0.5
#define ROULETTE_WEIGHT_CAP 4.0
#define QUANTUM 1.0e-9
#define INV_QUANTUM 1.0e9
#define ENTRY_NUDGE 1.0e-9
#define BOUNDARY_NUDGE 1.0e-4
#define HINGE_THETA2_MAX 0.10
#define GS_THETA2_MIN 1.0e-12
#define POLE_FLOOR 1.0e-20
#define STACK_CAP 4096

enum { PHOTON = 0, ELECTRON = 1, POSITRON = 2 };

typedef struct {
    int nx, ny, nz;
    double origin[3], spacing[3];
    const double* density;   /* [n] */
    const uint8_t* material; /* [n] */
} o_grid;

typedef struct {
    int n_materials, n_points;
    double p_log_min, p_inv_dlog, e_log_min, e_inv_dlog, r_log_min, r_inv_dlog;
    const double *mu_compton, *mu_photo, *mu_pair, *mu_rayleigh, *majorant;
    const double *stopping_radiative, *moller, *csda_range, *scattering_power, *log_eta;
    const double *restricted_range, *energy_of_restricted_range;
    int n_coherent;
    const double *coherent_x, *coherent_cumulative;
} o_tables;

typedef struct {
    const float* values; /* [n_eta][n_theta2][n_u] */
    int ix0, iy0, n_eta, n_theta2, n_u;
    double bins_per_log;
} o_gs;

/* Source of one call: forward (one column) or a Dij group of n_cols beamlets. */
typedef struct {
    int type; /* 0 pencil, 1 parallel/lattice, 2 spectral fan (optionally masked) */
    int kind; /* PHOTON or ELECTRON */
    double energy;
    double position[3], direction[3];
    double z0;
    const double *x_lo, *x_extent, *y_lo, *y_extent; /* [n_cols] */
    int n_bins;
    const double *edges, *cdf;
    double focal[3], u_axis[3], v_axis[3];
    double width_u, width_v;
    const double* centers; /* [n_cols][3] */
    /* spectral fan through a transmission mask (mask != NULL) */
    const double* mask; /* [mask_n_u][mask_n_v] */
    int mask_n_u, mask_n_v;
    double mask_center[3], mask_u[3], mask_v[3];
    double mask_width_u, mask_width_v;
} o_source;

/* _MaskTransmission.factors (geometry/collimation.py:1041-1080), one ray, in
 * float64: zero off the plane's rectangle or parallel to the plane, else the
 * clamped bilinear value between pixel centres. */
static double mask_factor(const o_source* s, const double p[3], const double d[3]) {
    const double* a = s->mask_u;
    const double* b = s->mask_v;
    const double n[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
    const double den = d[0] * n[0] + d[1] * n[1] + d[2] * n[2];
    if (den == 0.0) return 0.0;
    const double t = ((s->mask_center[0] - p[0]) * n[0] + (s->mask_center[1] - p[1]) * n[1] +
                      (s->mask_center[2] - p[2]) * n[2]) / den;
    double off[3];
    for (int k = 0; k < 3; ++k) off[k] = p[k] + t * d[k] - s->mask_center[k];
    const double u = off[0] * a[0] + off[1] * a[1] + off[2] * a[2];
    const double v = off[0] * b[0] + off[1] * b[1] + off[2] * b[2];
    if (!(fabs(u) <= s->mask_width_u / 2.0 && fabs(v) <= s->mask_width_v / 2.0)) return 0.0;
    const int nu = s->mask_n_u, nv = s->mask_n_v;
    double pu = (u + s->mask_width_u / 2.0) / (s->mask_width_u / nu) - 0.5;
    double pv = (v + s->mask_width_v / 2.0) / (s->mask_width_v / nv) - 0.5;
    pu = pu < 0.0 ? 0.0 : (pu > nu - 1 ? nu - 1 : pu);
    pv = pv < 0.0 ? 0.0 : (pv > nv - 1 ? nv - 1 : pv);
    int i0 = (int)pu, j0 = (int)pv;
    const int ci = nu - 2 > 0 ? nu - 2 : 0, cj = nv - 2 > 0 ? nv - 2 : 0;
    if (i0 > ci) i0 = ci;
    if (j0 > cj) j0 = cj;
    const int i1 = i0 + 1 < nu - 1 ? i0 + 1 : nu - 1;
    const int j1 = j0 + 1 < nv - 1 ? j0 + 1 : nv - 1;
    const double fu = pu - i0, fv = pv - j0;
    const double v00 = s->mask[i0 * nv + j0], v10 = s->mask[i1 * nv + j0];
    const double v01 = s->mask[i0 * nv + j1], v11 = s->mask[i1 * nv + j1];
    return v00 + fu * (v10 - v00) + fv * (v01 - v00) + fu * fv * (v11 - v10 - v01 + v00);
}

typedef struct {
    int forward;
    int n_cols;
    const int64_t* counts; /* [n_cols] histories per column */
    int n_batches;
    uint64_t seed;
    double pcut, ecut;
    int transport_electrons, msc_gs, correlated;
    double step_energy_fraction;
    int n_threads;
    int64_t first_history; /* forward: 0; Dij: global offset of column 0 */
    int64_t max_histories; /* > 0: transport only the first max_histories of each batch
                              (a bounded sample for timing; statistics then cover that) */
} o_params;

/* ---- Philox4x32-10 ---------------------------------------------------------- */
static void philox(uint32_t c[4], uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        if (r) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = (uint32_t)p1;
        c[2] = n2;
        c[3] = (uint32_t)p0;
    }
}

/* Known-answer check entry for the tests. */
void oracle_philox(const uint32_t counter[4], const uint32_t key[2], uint32_t out[4]) {
    memcpy(out, counter, 16);
    philox(out, key[0], key[1]);
}

typedef struct {
    uint32_t k0, k1, id0, id1;
    uint64_t block;
    uint32_t buf[4];
    int pos;
} rng_t;

static void rng_init(rng_t* r, uint64_t seed, uint64_t key) {
    r->k0 = (uint32_t)seed;
    r->k1 = (uint32_t)(seed >> 32);
    r->id0 = (uint32_t)key;
    r->id1 = (uint32_t)(key >> 32);
    r->block = 0;
    r->pos = 4;
}

static uint32_t rng_u32(rng_t* r) {
    if (r->pos == 4) {
        r->buf[0] = (uint32_t)r->block;
        r->buf[1] = r->id0;
        r->buf[2] = r->id1;
        r->buf[3] = (uint32_t)(r->block >> 32) | 0x80000000u; /* oracle namespace */
        philox(r->buf, r->k0, r->k1);
        r->block++;
        r->pos = 0;
    }
    return r->buf[r->pos++];
}

/* U[0, 1) with 53-bit resolution, like numpy's Generator.random(). */
static double uniform(rng_t* r) {
    uint64_t a = rng_u32(r) >> 5, b = rng_u32(r) >> 6;
    return (double)(a * 67108864ull + b) * (1.0 / 9007199254740992.0);
}

/* ---- geometry (geometry/grid.py) ---------------------------------------------- */
typedef struct {
    double lo[3], hi[3], sp[3];
    int n[3];
} box_t;

static int inside(const box_t* b, const double p[3]) {
    for (int a = 0; a < 3; ++a)
        if (p[a] < b->lo[a] || p[a] >= b->hi[a]) return 0;
    return 1;
}

static int axis_index(double p, double o, double s, int n) {
    int i = (int)floor((p - o) / s);
    if (i < 0) return 0;
    if (i >= n) return n - 1;
    return i;
}

static int64_t voxel(const box_t* b, const double p[3]) {
    int i[3];
    for (int a = 0; a < 3; ++a) i[a] = axis_index(p[a], b->lo[a], b->sp[a], b->n[a]);
    return ((int64_t)i[0] * b->n[1] + i[1]) * b->n[2] + i[2];
}

static double slab_entry(const box_t* b, const double p[3], const double u[3]) {
    double t_near = 0.0, t_far = INFINITY;
    for (int a = 0; a < 3; ++a) {
        if (u[a] == 0.0) {
            if (p[a] < b->lo[a] || p[a] >= b->hi[a]) return INFINITY;
        } else {
            double t1 = (b->lo[a] - p[a]) / u[a], t2 = (b->hi[a] - p[a]) / u[a];
            if (t1 > t2) {
                double t = t1;
                t1 = t2;
                t2 = t;
            }
            if (t1 > t_near) t_near = t1;
            if (t2 < t_far) t_far = t2;
        }
    }
    if (t_near > t_far || t_far <= 0.0) return INFINITY;
    return t_near;
}

static double boundary_distance(const box_t* b, const double p[3], const double u[3]) {
    double r = INFINITY;
    for (int a = 0; a < 3; ++a) {
        int i = axis_index(p[a], b->lo[a], b->sp[a], b->n[a]);
        double d;
        if (u[a] > 0.0) {
            d = (b->lo[a] + (double)(i + 1) * b->sp[a] - p[a]) / u[a];
            if (d < r) r = d;
        } else if (u[a] < 0.0) {
            d = (b->lo[a] + (double)i * b->sp[a] - p[a]) / u[a];
            if (d < r) r = d;
        }
    }
    return r > 0.0 ? r : 0.0;
}

/* ---- tables (data/tables.py:83-133) ------------------------------------------ */
static double lookup(const double* v, double log_min, double inv, int n, double q) {
    double t = (log(q) - log_min) * inv;
    if (t < 0.0) t = 0.0;
    if (t > (double)(n - 1)) t = (double)(n - 1);
    int i = (int)t;
    if (i > n - 2) i = n - 2;
    double w = t - (double)i;
    return v[i] * (1.0 - w) + v[i + 1] * w;
}

/* ---- physics samplers (physics/*.py) ------------------------------------------ */
static void rotate(double u[3], double cos_t, double phi) {
    double s = sqrt(fmax(0.0, 1.0 - cos_t * cos_t));
    double cp = cos(phi), sp = sin(phi);
    double t2 = u[0] * u[0] + u[1] * u[1];
    if (t2 > POLE_FLOOR) {
        double t = sqrt(t2), inv = s / t;
        double vx = u[0] * cos_t + inv * (u[0] * u[2] * cp - u[1] * sp);
        double vy = u[1] * cos_t + inv * (u[1] * u[2] * cp + u[0] * sp);
        double vz = u[2] * cos_t - t * s * cp;
        u[0] = vx;
        u[1] = vy;
        u[2] = vz;
        return;
    }
    double sign = u[2] > 0.0 ? 1.0 : -1.0;
    u[0] = s * cp;
    u[1] = sign * s * sp;
    u[2] = sign * cos_t;
}

static double kahn_ratio(double e, rng_t* r) {
    double alpha = e / ME, ta = 2.0 * alpha, bp = (1.0 + ta) / (9.0 + ta);
    for (;;) {
        double u1 = uniform(r), u2 = uniform(r), u3 = uniform(r);
        if (u1 <= bp) {
            double x = 1.0 + ta * u2;
            if (u3 <= 4.0 * (x - 1.0) / (x * x)) return 1.0 / x;
        } else {
            double x = (1.0 + ta) / (1.0 + ta * u2);
            double c = 1.0 - (x - 1.0) / alpha;
            if (u3 <= 0.5 * (c * c + 1.0 / x)) return 1.0 / x;
        }
    }
}

static double compton_cos(double e, double ratio) {
    double alpha = e / ME, c = 1.0 + 1.0 / alpha - 1.0 / (alpha * ratio);
    return fmin(1.0, fmax(-1.0, c));
}

static double compton_e_cos(double e, double ratio) {
    double recoil = e * (1.0 - ratio), p = sqrt(recoil * (recoil + 2.0 * ME));
    double c = (e - ratio * e * compton_cos(e, ratio)) / p;
    return fmin(1.0, fmax(-1.0, c));
}

static double moller_delta(double e, double cut, rng_t* r) {
    double tau = e / ME, tr = tau / (tau + 1.0), tr2 = tr * tr;
    double two = (2.0 * tau + 1.0) / ((tau + 1.0) * (tau + 1.0));
    double wmin = cut / e, bound = 2.0 + 0.25 * tr2;
    for (;;) {
        double u = uniform(r);
        double x = wmin / (1.0 - u * (1.0 - 2.0 * wmin));
        double q = x / (1.0 - x);
        double acc = 1.0 + q * q + x * x * tr2 - two * q;
        if (uniform(r) * bound <= acc) return x * e;
    }
}

static double interp_inc(double q, const double* xs, const double* ys, int n) {
    if (q <= xs[0]) return ys[0];
    if (q >= xs[n - 1]) return ys[n - 1];
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) {
        int mid = (lo + hi) / 2;
        if (xs[mid] <= q) lo = mid;
        else hi = mid;
    }
    double t = (q - xs[lo]) / (xs[hi] - xs[lo]);
    return ys[lo] * (1.0 - t) + ys[hi] * t;
}

typedef struct {
    int kind;
    double e, w, p[3], u[3];
} part_t;

typedef struct {
    const o_grid* g;
    const o_tables* t;
    const o_gs* gs;
    const o_params* P;
    box_t box;
    int64_t n_vox;
    int64_t* edep; /* [n_cols][n_vox] for the current batch */
    uint8_t* seen; /* [n_cols][n_vox] entry ever scored */
    int64_t* touched; /* indices of the entries ever scored */
    int64_t n_touched;
    int64_t escaped, deposited_unused, emitted;
    int error;
} ctx_t;

static void deposit(ctx_t* c, int col, const double p[3], double amount) {
    int64_t q = (int64_t)(amount * INV_QUANTUM + 0.5);
    if (q == 0) return;
    const int64_t idx = (int64_t)col * c->n_vox + voxel(&c->box, p);
    __atomic_fetch_add(c->edep + idx, q, __ATOMIC_RELAXED);
    if (!__atomic_load_n(c->seen + idx, __ATOMIC_RELAXED) &&
        !__atomic_exchange_n(c->seen + idx, (uint8_t)1, __ATOMIC_RELAXED))
        c->touched[__atomic_fetch_add(&c->n_touched, 1, __ATOMIC_RELAXED)] = idx;
}

static void escape(ctx_t* c, double amount) {
    int64_t q = (int64_t)floor(amount * INV_QUANTUM + 0.5);
    __atomic_fetch_add(&c->escaped, q, __ATOMIC_RELAXED);
}

static int push(part_t* stack, int* n, int kind, double e, double w, const double p[3],
                const double u[3], ctx_t* c) {
    if (*n >= STACK_CAP) {
        __atomic_store_n(&c->error, 1, __ATOMIC_RELAXED);
        return 0;
    }
    part_t* s = &stack[(*n)++];
    s->kind = kind;
    s->e = e;
    s->w = w;
    memcpy(s->p, p, sizeof s->p);
    memcpy(s->u, u, sizeof s->u);
    return 1;
}

static void annihilate(ctx_t* c, int col, const double p[3], double w, rng_t* r, part_t* stack,
                       int* n) {
    if (c->P->pcut >= ME) {
        deposit(c, col, p, w * 2.0 * ME);
        return;
    }
    double ct = 1.0 - 2.0 * uniform(r), st = sqrt(fmax(0.0, 1.0 - ct * ct));
    double phi = 2.0 * M_PI * uniform(r);
    double a[3] = {st * cos(phi), st * sin(phi), ct}, b[3] = {-a[0], -a[1], -a[2]};
    push(stack, n, PHOTON, ME, w, p, a, c);
    push(stack, n, PHOTON, ME, w, p, b, c);
}

/* photon_steps (transport/photon.py:100), unsplit (PHOTON_SPLIT_N = 1). */
static void photon_steps(ctx_t* c, int col, part_t* ph, rng_t* r, part_t* stack, int* n) {
    const o_tables* t = c->t;
    double e = ph->e, w = ph->w, p[3], u[3];
    memcpy(p, ph->p, sizeof p);
    memcpy(u, ph->u, sizeof u);
    if (!inside(&c->box, p)) {
        double d = slab_entry(&c->box, p, u);
        if (isinf(d)) {
            escape(c, w * e);
            return;
        }
        d += ENTRY_NUDGE;
        for (int a = 0; a < 3; ++a) p[a] += d * u[a];
        if (!inside(&c->box, p)) {
            escape(c, w * e);
            return;
        }
    }
    const double pcut = c->P->pcut, ecut = c->P->ecut;
    for (long steps = 0; steps < 100000000L; ++steps) {
        double maj = lookup(t->majorant, t->p_log_min, t->p_inv_dlog, t->n_points, e);
        double s = -log1p(-uniform(r)) / maj;
        for (int a = 0; a < 3; ++a) p[a] += s * u[a];
        if (!inside(&c->box, p)) {
            escape(c, w * e);
            return;
        }
        int64_t v = voxel(&c->box, p);
        double rho = c->g->density[v];
        int mat = c->g->material[v];
        const int64_t row = (int64_t)mat * t->n_points;
        double mc = rho * lookup(t->mu_compton + row, t->p_log_min, t->p_inv_dlog, t->n_points, e);
        double mp = rho * lookup(t->mu_photo + row, t->p_log_min, t->p_inv_dlog, t->n_points, e);
        double mpa = rho * lookup(t->mu_pair + row, t->p_log_min, t->p_inv_dlog, t->n_points, e);
        double mr = rho * lookup(t->mu_rayleigh + row, t->p_log_min, t->p_inv_dlog, t->n_points, e);
        double real = mc + mp + mpa + mr;
        if (real > maj * (1.0 + 1.0e-9)) {
            __atomic_store_n(&c->error, 2, __ATOMIC_RELAXED);
            escape(c, w * e);
            return;
        }
        if (uniform(r) * maj >= real) continue;
        double thr = uniform(r) * (mc + mp + mpa + mr);
        if (thr >= mc + mp + mpa) { /* coherent (form-factor sampler, physics/rayleigh.py:43) */
            const double* cum = t->coherent_cumulative + (int64_t)mat * t->n_coherent;
            double xm = 80.65543 * e, am = interp_inc(xm, t->coherent_x, cum, t->n_coherent), mu;
            for (;;) {
                double x = interp_inc(uniform(r) * am, cum, t->coherent_x, t->n_coherent);
                double rat = x / xm;
                mu = 1.0 - 2.0 * rat * rat;
                if (2.0 * uniform(r) <= 1.0 + mu * mu) break;
            }
            rotate(u, mu, 2.0 * M_PI * uniform(r));
            continue;
        }
        if (thr < mc) { /* Compton: the scattered photon goes back on the stack */
            double ratio = kahn_ratio(e, r), recoil = e * (1.0 - ratio);
            double phi = 2.0 * M_PI * uniform(r);
            if (c->P->transport_electrons && recoil > ecut) {
                double eu[3] = {u[0], u[1], u[2]};
                rotate(eu, compton_e_cos(e, ratio), phi + M_PI);
                push(stack, n, ELECTRON, recoil, w, p, eu, c);
            } else {
                deposit(c, col, p, w * recoil);
            }
            double gu[3] = {u[0], u[1], u[2]};
            rotate(gu, compton_cos(e, ratio), phi);
            double es = e * ratio;
            if (es <= pcut) {
                deposit(c, col, p, w * es);
                return;
            }
            double cw = w;
            if (es < ROULETTE_MEV && cw < ROULETTE_WEIGHT_CAP) {
                double nw = uniform(r) < ROULETTE_SURVIVAL ? cw / ROULETTE_SURVIVAL : 0.0;
                escape(c, (cw - nw) * es);
                if (nw == 0.0) return;
                cw = nw;
            }
            push(stack, n, PHOTON, es, cw, p, gu, c);
            return;
        }
        if (thr < mc + mp) { /* photoelectric */
            if (c->P->transport_electrons && e > ecut) push(stack, n, ELECTRON, e, w, p, u, c);
            else deposit(c, col, p, w * e);
            return;
        }
        /* pair */
        double kin = e - 2.0 * ME;
        if (c->P->transport_electrons) {
            double f = uniform(r);
            double se = f * kin, sp = (1.0 - f) * kin;
            if (se > ecut) push(stack, n, ELECTRON, se, w, p, u, c);
            else deposit(c, col, p, w * se);
            if (sp > ecut) {
                push(stack, n, POSITRON, sp, w, p, u, c);
            } else {
                deposit(c, col, p, w * sp);
                annihilate(c, col, p, w, r, stack, n);
            }
        } else {
            deposit(c, col, p, w * kin);
            annihilate(c, col, p, w, r, stack, n);
        }
        return;
    }
    __atomic_store_n(&c->error, 3, __ATOMIC_RELAXED);
}

static double deposit_or_escape(ctx_t* c, int col, const double p[3], double amount) {
    if (amount <= 0.0) return 0.0;
    if (inside(&c->box, p)) {
        deposit(c, col, p, amount);
        return 0.0;
    }
    return amount;
}

static double gs_sample(const o_gs* g, double fx, double fy, double ms, rng_t* r) {
    int ix = (int)floor(fx) - g->ix0, iy = (int)floor(fy) - g->iy0;
    if (ix < 0) ix = 0;
    if (ix > g->n_eta - 2) ix = g->n_eta - 2;
    if (iy < 0) iy = 0;
    if (iy > g->n_theta2 - 2) iy = g->n_theta2 - 2;
    double tx = fmin(fmax(fx - (double)(g->ix0 + ix), 0.0), 1.0);
    double ty = fmin(fmax(fy - (double)(g->iy0 + iy), 0.0), 1.0);
    if (ms <= 0.0) return 1.0;
    int k = (int)(uniform(r) * (double)g->n_u);
    if (k > g->n_u - 1) k = g->n_u - 1;
#define GSV(i, j) ((double)g->values[((int64_t)(i) * g->n_theta2 + (j)) * g->n_u + k])
    double lo = GSV(ix, iy) * (1.0 - tx) + GSV(ix + 1, iy) * tx;
    double hi = GSV(ix, iy + 1) * (1.0 - tx) + GSV(ix + 1, iy + 1) * tx;
#undef GSV
    double wv = lo * (1.0 - ty) + hi * ty;
    return fmax(-1.0, 1.0 - wv * (-expm1(-0.5 * ms)));
}

/* electron_steps (transport/electron.py:207), single midpoint deposits. */
static void electron_steps(ctx_t* c, int col, part_t* el, rng_t* r, part_t* stack, int* n) {
    const o_tables* t = c->t;
    const int positron = el->kind == POSITRON;
    double e = el->e, w = el->w, p[3], u[3];
    memcpy(p, el->p, sizeof p);
    memcpy(u, el->u, sizeof u);
    const double latent = positron ? 2.0 * ME : 0.0;
    const double pcut = c->P->pcut, ecut = c->P->ecut;
    if (!inside(&c->box, p)) {
        double d = slab_entry(&c->box, p, u);
        if (isinf(d)) {
            escape(c, w * (e + latent));
            return;
        }
        d += ENTRY_NUDGE;
        for (int a = 0; a < 3; ++a) p[a] += d * u[a];
        if (!inside(&c->box, p)) {
            escape(c, w * (e + latent));
            return;
        }
    }
    for (long steps = 0; steps < 100000000L; ++steps) {
        if (e <= ecut) {
            deposit(c, col, p, w * e);
            if (positron) annihilate(c, col, p, w, r, stack, n);
            return;
        }
        int64_t v = voxel(&c->box, p);
        double rho = c->g->density[v];
        int mat = c->g->material[v];
        const int64_t row = (int64_t)mat * t->n_points;
#define EL(tab, q) lookup((tab) + row, t->e_log_min, t->e_inv_dlog, t->n_points, (q))
        double range_cm = EL(t->csda_range, e) / rho;
        double s_max = c->P->step_energy_fraction * range_cm;
        if (!c->P->msc_gs) {
            double st = HINGE_THETA2_MAX / (EL(t->scattering_power, e) * rho);
            if (st < s_max) s_max = st;
        }
        double s_b = boundary_distance(&c->box, p, u) + BOUNDARY_NUDGE;
        double s_geo = fmin(s_max, s_b);
        double sig = rho * EL(t->moller, e);
        double s_int = sig > 0.0 ? -log1p(-uniform(r)) / sig : INFINITY;
        double s = fmin(s_int, s_geo);
        int pending = s_int <= s_geo;
        double avail = EL(t->restricted_range, e), de;
        if (rho * s >= avail) {
            s = avail / rho;
            de = e - ecut;
            pending = 0;
        } else {
            double e_end = lookup(t->energy_of_restricted_range + row, t->r_log_min, t->r_inv_dlog,
                                  t->n_points, avail - rho * s);
            e_end = fmin(fmax(e_end, ecut), e);
            de = e - e_end;
        }
        double srad = EL(t->stopping_radiative, e), loss = srad * rho * s, prob, local;
        if (e <= pcut) {
            prob = 0.0;
            local = loss;
        } else {
            double frac = 1.0 - pcut / e, mk = (e - pcut) / log(e / pcut);
            prob = loss * frac / mk;
            local = loss * (1.0 - frac);
        }
        double cont = de + local;
        int emit = uniform(r) < prob;
        double s1 = uniform(r) * s, s2 = s - s1;
        double d1 = s > 0.0 ? cont * (s1 / s) : 0.0, d2 = cont - d1;
        double mid[3];
        for (int a = 0; a < 3; ++a) mid[a] = p[a] + u[a] * (0.5 * s1);
        double esc = deposit_or_escape(c, col, mid, w * d1);
        if (esc != 0.0) escape(c, esc);
        e -= d1;
        for (int a = 0; a < 3; ++a) p[a] += u[a] * s1;
        if (!inside(&c->box, p)) {
            escape(c, w * (e + latent));
            return;
        }
        double ms = EL(t->scattering_power, e) * rho * s, ch;
        if (c->P->msc_gs) {
            double fx = EL(t->log_eta, e) * c->gs->bins_per_log;
            double fy = log(fmax(ms, GS_THETA2_MIN)) * c->gs->bins_per_log;
            ch = gs_sample(c->gs, fx, fy, ms, r);
        } else {
            double th = sqrt(-ms * log1p(-uniform(r)));
            ch = cos(fmin(th, M_PI));
        }
#undef EL
        rotate(u, ch, 2.0 * M_PI * uniform(r));
        if (emit && e > pcut) {
            double k = pcut * exp(uniform(r) * log(e / pcut));
            if (k > e - d2) k = e - d2;
            if (k > pcut) {
                double pw = w;
                if (k < ROULETTE_MEV && w < ROULETTE_WEIGHT_CAP) {
                    pw = uniform(r) < ROULETTE_SURVIVAL ? w / ROULETTE_SURVIVAL : 0.0;
                    escape(c, (w - pw) * k);
                }
                if (pw > 0.0) push(stack, n, PHOTON, k, pw, p, u, c);
            } else {
                double x = deposit_or_escape(c, col, p, w * k);
                if (x != 0.0) escape(c, x);
            }
            e -= k;
        }
        for (int a = 0; a < 3; ++a) mid[a] = p[a] + u[a] * (0.5 * s2);
        esc = deposit_or_escape(c, col, mid, w * d2);
        if (esc != 0.0) escape(c, esc);
        e -= d2;
        for (int a = 0; a < 3; ++a) p[a] += u[a] * s2;
        if (!inside(&c->box, p)) {
            escape(c, w * (e + latent));
            return;
        }
        if (pending && e > 2.0 * ecut) {
            double wd = moller_delta(e, ecut, r);
            double two = 2.0 * ME, rest = e - wd;
            double cd = fmin(1.0, sqrt(wd * (e + two) / (e * (wd + two))));
            double cp = fmin(1.0, sqrt(rest * (e + two) / (e * (rest + two))));
            double phi = 2.0 * M_PI * uniform(r);
            double du[3] = {u[0], u[1], u[2]};
            rotate(du, cd, phi);
            push(stack, n, ELECTRON, wd, w, p, du, c);
            rotate(u, cp, phi + M_PI);
            e -= wd;
        }
    }
    __atomic_store_n(&c->error, 3, __ATOMIC_RELAXED);
}

/* One primary of column col: sample it (geometry/source.py emit) and transport
 * the family (transport/history.py:31). */
static void history(ctx_t* c, const o_source* s, int col, uint64_t key) {
    rng_t r;
    rng_init(&r, c->P->seed, key);
    part_t stack[STACK_CAP];
    int n = 0;
    part_t pr;
    pr.kind = s->kind;
    pr.w = 1.0;
    if (s->type == 0) {
        pr.e = s->energy;
        memcpy(pr.p, s->position, sizeof pr.p);
        memcpy(pr.u, s->direction, sizeof pr.u);
    } else if (s->type == 1) {
        pr.e = s->energy;
        pr.p[0] = s->x_lo[col] + s->x_extent[col] * uniform(&r);
        pr.p[1] = s->y_lo[col] + s->y_extent[col] * uniform(&r);
        pr.p[2] = s->z0;
        pr.u[0] = 0.0;
        pr.u[1] = 0.0;
        pr.u[2] = 1.0;
    } else {
        double ub = uniform(&r);
        int lo = 0, hi = s->n_bins;
        while (lo < hi) {
            int mid = (lo + hi) / 2;
            if (s->cdf[mid] < ub) lo = mid + 1;
            else hi = mid;
        }
        int k = lo < s->n_bins - 1 ? lo : s->n_bins - 1;
        pr.e = s->edges[k] + (s->edges[k + 1] - s->edges[k]) * uniform(&r);
        double du = (uniform(&r) - 0.5) * s->width_u, dv = (uniform(&r) - 0.5) * s->width_v;
        double d[3], norm = 0.0;
        for (int a = 0; a < 3; ++a) {
            d[a] = s->centers[3 * col + a] + du * s->u_axis[a] + dv * s->v_axis[a] - s->focal[a];
            norm += d[a] * d[a];
        }
        norm = sqrt(norm);
        for (int a = 0; a < 3; ++a) pr.u[a] = d[a] / norm;
        memcpy(pr.p, s->focal, sizeof pr.p);
        pr.kind = PHOTON;
        if (s->mask) {  /* TransmissionMaskSource: a zero factor emits nothing */
            pr.w = mask_factor(s, pr.p, pr.u);
            if (pr.w == 0.0) return;
        }
        int64_t q = (int64_t)floor(pr.w * pr.e * INV_QUANTUM + 0.5);
        __atomic_fetch_add(&c->emitted, q, __ATOMIC_RELAXED);
    }
    stack[n++] = pr;
    while (n > 0) {
        part_t cur = stack[--n];
        if (cur.kind == PHOTON) photon_steps(c, col, &cur, &r, stack, &n);
        else electron_steps(c, col, &cur, &r, stack, &n);
    }
}

typedef struct {
    ctx_t* c;
    const o_source* s;
    int batch, n_cols;
    const int64_t* per_batch; /* [n_cols] */
    const int64_t* prefix;    /* [n_cols+1] exclusive prefix of the sampled counts */
    const int64_t* col_offset; /* [n_cols] first global history of each column */
    int64_t total;
    int64_t next; /* shared work counter */
} work_t;

static void* worker(void* arg) {
    work_t* w = (work_t*)arg;
    const o_params* P = w->c->P;
    for (;;) {
        int64_t t0 = __atomic_fetch_add(&w->next, 64, __ATOMIC_RELAXED);
        if (t0 >= w->total) break;
        int64_t t1 = t0 + 64 < w->total ? t0 + 64 : w->total;
        for (int64_t t = t0; t < t1; ++t) {
            int lo = 0, hi = w->n_cols; /* largest column with prefix[col] <= t */
            while (hi - lo > 1) {
                int mid = (lo + hi) / 2;
                if (w->prefix[mid] <= t) lo = mid;
                else hi = mid;
            }
            const int col = lo;
            const int64_t i = t - w->prefix[col];
            int64_t rr = (int64_t)w->batch * w->per_batch[col] + i;
            int64_t h = P->forward ? rr : w->col_offset[col] + rr;
            uint64_t key = (!P->forward && P->correlated) ? (uint64_t)rr : (uint64_t)h;
            history(w->c, w->s, col, key);
        }
    }
    return NULL;
}

/*
 * Transport every column's histories in batch order, fold each batch's quanta
 * into float64 batch sums, and finalize mean and sigma per entry.  mean and
 * sigma are [n_cols][n_vox] and must arrive zeroed (only scored entries are
 * written).  books = {deposited, escaped, emitted} quanta.
 * Returns 0, or 1 stack overflow / 2 majorant violation / 3 step cap.
 */
int oracle_transport(const o_grid* g, const o_tables* t, const o_gs* gs, const o_source* s,
                     const o_params* P, double* mean, double* sigma, int64_t books[3]) {
    ctx_t c;
    memset(&c, 0, sizeof c);
    c.g = g;
    c.t = t;
    c.gs = gs;
    c.P = P;
    const int nn[3] = {g->nx, g->ny, g->nz};
    for (int a = 0; a < 3; ++a) {
        c.box.lo[a] = g->origin[a];
        c.box.hi[a] = g->origin[a] + nn[a] * g->spacing[a];
        c.box.sp[a] = g->spacing[a];
        c.box.n[a] = nn[a];
    }
    c.n_vox = (int64_t)g->nx * g->ny * g->nz;
    const int64_t span = c.n_vox * P->n_cols;
    /* calloc'd pages are zero-filled lazily, so only scored entries cost memory */
    c.edep = (int64_t*)calloc((size_t)span, sizeof(int64_t));
    c.seen = (uint8_t*)calloc((size_t)span, 1);
    c.touched = (int64_t*)calloc((size_t)span, sizeof(int64_t));
    double* s1 = (double*)calloc((size_t)span, sizeof(double));
    double* s2 = (double*)calloc((size_t)span, sizeof(double));
    if (!c.edep || !c.seen || !c.touched || !s1 || !s2) {
        free(c.edep);
        free(c.seen);
        free(c.touched);
        free(s1);
        free(s2);
        return 4;
    }
    int n_threads = P->n_threads > 0 ? P->n_threads : 1;
    if (n_threads > 512) n_threads = 512;
    pthread_t threads[512];
    pthread_attr_t attr;
    pthread_attr_init(&attr);
    pthread_attr_setstacksize(&attr, 8u << 20);
    const double vol = g->spacing[0] * g->spacing[1] * g->spacing[2];
    int64_t deposited = 0;
    const int nc = P->n_cols;
    int64_t* per_batch = (int64_t*)calloc((size_t)nc, sizeof(int64_t));
    int64_t* prefix = (int64_t*)calloc((size_t)nc + 1, sizeof(int64_t));
    int64_t* offs = (int64_t*)calloc((size_t)nc, sizeof(int64_t));
    double* nh = (double*)calloc((size_t)nc, sizeof(double));
    int64_t acc = P->first_history;
    for (int col = 0; col < nc; ++col) {
        per_batch[col] = P->counts[col] / P->n_batches;
        int64_t todo = per_batch[col];
        if (P->max_histories > 0 && todo > P->max_histories) todo = P->max_histories;
        prefix[col + 1] = prefix[col] + todo;
        nh[col] = (double)todo;
        offs[col] = acc;
        acc += P->counts[col];
    }
    for (int b = 0; b < P->n_batches; ++b) {
        work_t w;
        w.c = &c;
        w.s = s;
        w.batch = b;
        w.n_cols = nc;
        w.per_batch = per_batch;
        w.prefix = prefix;
        w.col_offset = offs;
        w.total = prefix[nc];
        w.next = 0;
        int started = 0;
        for (int k = 1; k < n_threads; ++k)
            if (pthread_create(&threads[k], &attr, worker, &w) == 0) ++started;
            else break;
        worker(&w);
        for (int k = 1; k <= started; ++k) pthread_join(threads[k], NULL);
        /* fold (scoring/dij.py:155-174): dose = E / (mass * n), over the entries
         * scored so far (an unscored entry adds +0.0 and changes nothing) */
        for (int64_t k = 0; k < c.n_touched; ++k) {
            const int64_t idx = c.touched[k];
            const int64_t q = c.edep[idx];
            if (q == 0) continue;
            c.edep[idx] = 0;
            deposited += q;
            const int64_t col = idx / c.n_vox;
            const double m = g->density[idx - col * c.n_vox] * vol;
            const double d = m > 0.0 ? ((double)q * QUANTUM) / (m * nh[col]) : 0.0;
            s1[idx] += d;
            s2[idx] += d * d;
        }
    }
    free(per_batch);
    free(prefix);
    free(offs);
    free(nh);
    pthread_attr_destroy(&attr);
    const double n = (double)P->n_batches;
    for (int64_t k = 0; k < c.n_touched; ++k) { /* mean, sigma of untouched entries stay 0 */
        const int64_t i = c.touched[k];
        double m = s1[i] / n, sg = 0.0;
        if (P->n_batches > 1) {
            double var = s2[i] / n - m * m;
            if (var < 0.0) var = 0.0;
            sg = sqrt((var * n / (n - 1.0)) / n);
        }
        mean[i] = m;
        sigma[i] = sg;
    }
    books[0] = deposited;
    books[1] = c.escaped;
    books[2] = c.emitted;
    free(c.edep);
    free(c.seen);
    free(c.touched);
    free(s1);
    free(s2);
    return c.error;
}

int oracle_max_threads(void) {
    long n = sysconf(_SC_NPROCESSORS_ONLN);
    return n > 0 ? (int)n : 1;
}
