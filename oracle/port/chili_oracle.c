/*
 * chili_oracle.c -- CPU restatement, in plain C, of Chili's VEGAS +
 * multichannel FSMapper hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  It is the checker for the CUDA library: tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg call it; the
 * product never links it.  It is pinned against the reference itself
 * (oracle/_ref, the unmodified sources) by tests/test_oracle_pin.py and the
 * committed fixtures in tests/golden/.
 *
 * Every function cites the reference file:line (paths inside the Chili
 * project) whose arithmetic it restates; operations keep the reference's
 * order, and the file is compiled with -ffp-contract=off like the reference
 * (no FMA on x86-64 by default).  Channel descriptions and cuts come in the
 * flat structs of include/chili_gpu.h.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "chili_gpu.h"

#define PI 3.14159265358979323846
#define DBL_MAXV 1.7976931348623157e308
#define DBL_MINV 2.2250738585072014e-308

static double dmin_(double a, double b) { return (b < a) ? b : a; } /* std::min */
static double dmax_(double a, double b) { return (a < b) ? b : a; } /* std::max */

/* ------------------------------------------------------------------ Philox */
/* Philox4x32-10 (Salmon et al., SC'11) and the 53-bit uniform the CUDA
 * library draws for point k, uniform j: block {j/2, lo(k), hi(k), 0}, key
 * {lo(seed), hi(seed)}, words (0,1) -> uniform 2q, (2,3) -> 2q+1. */
static void philox(uint32_t c[4], uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c[0], p1 = (uint64_t)0xCD9E8D57u * c[2];
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0, n1 = (uint32_t)p1;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1, n3 = (uint32_t)p0;
        c[0] = n0; c[1] = n1; c[2] = n2; c[3] = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}
static double u53(uint32_t hi, uint32_t lo) {
    return (double)(((uint64_t)hi << 21) | (lo >> 11)) * 0x1.0p-53;
}
/* Stream s of the same generator: block word 3 = s (0: the points, 1: the
 * unweighting stage's accept uniforms). */
void orc_philox_stream_uniforms(uint64_t seed, uint64_t ctr0, int64_t n, int d, uint32_t stream, double *out) {
    for (int64_t i = 0; i < n; ++i) {
        uint64_t k = ctr0 + (uint64_t)i;
        for (int q = 0; 2 * q < d; ++q) {
            uint32_t c[4] = {(uint32_t)q, (uint32_t)k, (uint32_t)(k >> 32), stream};
            philox(c, (uint32_t)seed, (uint32_t)(seed >> 32));
            out[i * d + 2 * q] = u53(c[0], c[1]);
            if (2 * q + 1 < d) out[i * d + 2 * q + 1] = u53(c[2], c[3]);
        }
    }
}
void orc_philox_uniforms(uint64_t seed, uint64_t ctr0, int64_t n, int d, double *out) {
    for (int64_t i = 0; i < n; ++i) {
        uint64_t k = ctr0 + (uint64_t)i;
        for (int q = 0; 2 * q < d; ++q) {
            uint32_t c[4] = {(uint32_t)q, (uint32_t)k, (uint32_t)(k >> 32), 0u};
            philox(c, (uint32_t)seed, (uint32_t)(seed >> 32));
            out[i * d + 2 * q] = u53(c[0], c[1]);
            if (2 * q + 1 < d) out[i * d + 2 * q + 1] = u53(c[2], c[3]);
        }
    }
}

/* ------------------------------------------------------------- AdaptiveMap */
/* FindBin (AdaptiveMap.cc:34-38): lower_bound over the first `bins` edges
 * minus one; -1 stands for the reference's SIZE_MAX. */
static int find_bin(const double *e, int bins, double x) {
    int first = 0, len = bins;
    while (len > 0) {
        int half = len >> 1, mid = first + half;
        if (e[mid] < x) { first = mid + 1; len = len - half - 1; }
        else len = half;
    }
    return first - 1;
}
/* The word in front of the reference's edge vector, read by width(0,
 * SIZE_MAX) (AdaptiveMap.hh:47-49): under glibc malloc the chunk size of the
 * buffer, (request + 8) rounded up to 16 with PREV_INUSE set (page-rounded
 * with IS_MMAPPED from 128 KiB up), i.e. a positive denormal as a double. */
static double before_table(int dims, int bins) {
    uint64_t req = 8ull * (uint64_t)dims * (uint64_t)(bins + 1), w;
    if (req + 8 >= 128ull * 1024) w = ((req + 16 + 4095) & ~4095ull) | 2ull;
    else {
        w = (req + 8 + 15) & ~15ull;
        if (w < 32) w = 32;
        w |= 1ull;
    }
    double d;
    memcpy(&d, &w, sizeof d);
    return d;
}
/* width(dim, bin) on the flat table, bin -1 reading the flat index before
 * the dimension: the previous dimension's last edge, or before_table(). */
static double width_(const double *g, int dims, int bins, int d, int b) {
    int base = d * (bins + 1);
    if (b >= 0) return g[base + b + 1] - g[base + b];
    return g[base] - (d > 0 ? g[base - 1] : before_table(dims, bins));
}
/* operator() (AdaptiveMap.cc:40-56); returns 0 when a uniform is outside [0,1) */
static int am_map1(const double *g, int dims, int bins, double *x, double *jac) {
    double j = 1.0;
    for (int i = 0; i < dims; ++i) {
        double pos = x[i] * (double)bins;
        if (!(pos >= 0.0 && pos < (double)bins)) return 0;
        int idx = (int)pos;
        double loc = pos - (double)idx;
        double left = g[i * (bins + 1) + idx];
        double size = g[i * (bins + 1) + idx + 1] - left;
        x[i] = left + loc * size;
        j *= size * (double)bins;
    }
    *jac = j;
    return 1;
}
/* GenerateWeight (AdaptiveMap.cc:58-65) */
static double am_weight1(const double *g, int dims, int bins, const double *x) {
    double j = 1.0;
    for (int i = 0; i < dims; ++i) j *= width_(g, dims, bins, i, find_bin(g + i * (bins + 1), bins, x[i])) * (double)bins;
    return j;
}
/* Adapt (AdaptiveMap.cc:67-125) of one grid; returns 1 if the rebinning ran
 * outside the histogram (undefined in the reference). */
static int am_adapt1(double *g, int dims, int bins, double alpha, const double *data) {
    double *tmp = malloc(sizeof(double) * bins);
    double *nh = calloc((size_t)dims * (bins + 1), sizeof(double));
    int bad = 0;
    for (int i = 0; i < dims; ++i) {
        memcpy(tmp, data + i * bins, sizeof(double) * bins);
        double prev = tmp[0], cur = tmp[1];
        tmp[0] = (prev + cur) / 2;
        double norm = tmp[0];
        for (int b = 1; b < bins - 1; ++b) {
            double sum = prev + cur;
            prev = cur;
            cur = tmp[b + 1];
            tmp[b] = (sum + cur) / 3;
            norm += tmp[b];
        }
        tmp[bins - 1] = (prev + cur) / 2;
        norm += tmp[bins - 1];
        if (norm == 0) continue;
        double avg = 0;
        for (int b = 0; b < bins; ++b)
            if (tmp[b] != 0) {
                double r = tmp[b] / norm;
                double fac = pow((r - 1.0) / log(r), alpha);
                avg += fac;
                tmp[b] = fac;
            }
        avg /= (double)bins;
        double cbin = 0;
        int ibin = 0;
        for (int nb = 1; nb < bins; ++nb) {
            while (cbin < avg && ibin < bins) cbin += tmp[ibin++];
            if (cbin < avg || ibin == 0) bad = 1;
            int fp = i * (bins + 1) + ibin - 1;
            double pv = fp >= 0 ? g[fp] : NAN;
            double cv = g[i * (bins + 1) + ibin];
            cbin -= avg;
            double delta = (cv - pv) * cbin;
            nh[i * (bins + 1) + nb] = cv - delta / (ibin > 0 ? tmp[ibin - 1] : NAN);
        }
        nh[i * (bins + 1) + bins] = 1.0;
    }
    memcpy(g, nh, sizeof(double) * dims * (bins + 1));
    free(tmp);
    free(nh);
    return bad;
}

void orc_am_map(int dims, int bins, const double *edges, const double *u, int64_t n, double *x, double *jac) {
    for (int64_t i = 0; i < n; ++i) {
        memcpy(x + i * dims, u + i * dims, sizeof(double) * dims);
        if (!am_map1(edges, dims, bins, x + i * dims, jac + i)) {
            for (int d = 0; d < dims; ++d) x[i * dims + d] = NAN;
            jac[i] = NAN;
        }
    }
}
void orc_am_weight(int dims, int bins, const double *edges, const double *x, int64_t n, double *w, int32_t *bin) {
    for (int64_t i = 0; i < n; ++i) {
        for (int d = 0; d < dims; ++d)
            if (bin) bin[i * dims + d] = find_bin(edges + d * (bins + 1), bins, x[i * dims + d]);
        if (w) w[i] = am_weight1(edges, dims, bins, x + i * dims);
    }
}
int orc_am_adapt(int dims, int bins, const double *edges, double alpha, const double *train, double *out) {
    memcpy(out, edges, sizeof(double) * dims * (bins + 1));
    return am_adapt1(out, dims, bins, alpha, train);
}
/* Split (AdaptiveMap.cc:127-160) */
void orc_am_split(int dims, int bins, const double *e, int nsplit, double *out) {
    int nb = nsplit * bins;
    for (int d = 0; d < dims; ++d) {
        for (int b = 0; b < bins; ++b) {
            double cur = e[d * (bins + 1) + b];
            double size = e[d * (bins + 1) + b + 1] - cur;
            for (int i = 0; i < nsplit; ++i) out[d * (nb + 1) + b * nsplit + i] = cur + (double)i * size / (double)nsplit;
        }
        out[d * (nb + 1) + nb] = 1.0;
    }
}

/* ------------------------------------------------------------- StatsData */
typedef struct { double n, mn, mx, sum, sum2, nf; } stats_t; /* Statistics.hh:62-142 */
static void st_init(stats_t *s) { s->n = 0; s->mn = DBL_MAXV; s->mx = DBL_MINV; s->sum = 0; s->sum2 = 0; s->nf = 0; }
static void st_add(stats_t *s, double x) {
    s->n++;
    s->sum += x;
    s->sum2 += x * x;
    s->mn = dmin_(s->mn, x);
    s->mx = dmax_(s->mx, x);
    if (x != 0) s->nf++;
}
static void st_out(const stats_t *s, chili_stats *o) {
    o->n = s->n; o->min = s->mn; o->max = s->mx; o->sum = s->sum; o->sum2 = s->sum2; o->n_finite = s->nf;
}

/* ------------------------------------------------------------- integrands */
static double camel(const double *p, const double *x, int d) {
    double s = p[0], norm = p[1], d1 = 0, d2 = 0;
    for (int i = 0; i < d; ++i) {
        double t = x[i] - p[2 + i];
        d1 += t * t;
        t = x[i] - p[2 + d + i];
        d2 += t * t;
    }
    double s2 = s * s;
    return norm * (exp(-d1 / s2) + exp(-d2 / s2));
}

typedef struct { double e, x, y, z; } v4;
static v4 vadd(v4 a, v4 b) { v4 r = {a.e + b.e, a.x + b.x, a.y + b.y, a.z + b.z}; return r; }
static v4 vsub(v4 a, v4 b) { v4 r = {a.e - b.e, a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static v4 vmul(v4 a, double s) { v4 r = {a.e * s, a.x * s, a.y * s, a.z * s}; return r; }
static double mdot(v4 a, v4 b) { return a.e * b.e - (a.x * b.x + a.y * b.y + a.z * b.z); } /* FourVector.cc:169-172 */
static double m2_(v4 a) { return mdot(a, a); }
static double pt2_(v4 a) { return a.x * a.x + a.y * a.y; }
static double p2_(v4 a) { return pt2_(a) + a.z * a.z; }
static double dot3_(v4 a, v4 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static double rap_(v4 a) { /* FourVector.cc:26-29 */
    if (a.e == 0) return 99;
    return log((a.e + a.z) / (a.e - a.z)) / 2;
}
static double phi_(v4 a) { /* FourVector.cc:20-24 */
    double p = atan2(a.y, a.x);
    return p < 0 ? p + 2 * PI : p;
}

static double propagator(const double *p, const v4 *mom, int n, int top2) {
    double m2 = p[0] * p[0], mw2 = p[0] * p[0] * p[1] * p[1], mt2 = p[2] * p[2];
    double sum = 0, b1 = 0, b2 = 0;
    for (int i = 2; i < n; ++i)
        for (int j = i + 1; j < n; ++j) {
            double d = m2_(vadd(mom[i], mom[j])) - m2;
            double bw = 1.0 / (d * d + mw2);
            sum += bw;
            if (bw > b1) { b2 = b1; b1 = bw; }
            else if (bw > b2) b2 = bw;
        }
    double t = 1;
    for (int j = 2; j < n; ++j) t *= 1.0 / (fabs(m2_(vadd(mom[0], mom[j]))) + mt2);
    return (top2 ? b1 * b2 : sum) * t;
}

/* ------------------------------------------------------ channel elements */
static double sqlam(double s, double s1, double s2) { /* ChannelElements.cc:21-25 */
    double a = s - s1 - s2, arg = a * a - 4. * s1 * s2;
    return arg > 0. ? sqrt(arg) / s : 0.;
}
/* PeakedDist/PeakedWeight with a=0, k=1 (ChannelElements.cc:27-62) */
static double ml_mom(double cn, double lo, double hi, double r) {
    double ce = 1. - cn;
    if (ce != 0.) return pow(r * pow(hi, ce) + (1. - r) * pow(lo, ce), 1 / ce);
    return lo * pow(hi / lo, r);
}
static double ml_wgt(double cn, double lo, double hi, double s, double *r) {
    double ce = 1. - cn, w;
    if (ce != 0.) {
        double amin = pow(lo, ce);
        w = pow(hi, ce) - amin;
        *r = (pow(s, ce) - amin) / w;
        w /= ce;
    } else {
        w = log(hi / lo);
        *r = log(s / lo) / w;
    }
    return w / pow(s, -cn);
}
/* Breit-Wigner (ChannelElements.cc:64-85) */
static double bw_mom(double m, double g, double lo, double hi, double r) {
    double m2 = m * m, mw = m * g, ymax = atan((lo - m2) / mw), ymin = atan((hi - m2) / mw);
    return m2 + mw * tan(ymin + r * (ymax - ymin));
}
static double bw_wgt(double m, double g, double lo, double hi, double s, double *r) {
    double m2 = m * m, mw = m * g, ymax = atan((lo - m2) / mw), ymin = atan((hi - m2) / mw);
    double y = atan((s - m2) / mw);
    *r = (y - ymin) / (ymax - ymin);
    double w = mw / ((s - m2) * (s - m2) + mw * mw);
    return (ymin - ymax) / w;
}
/* LT (ChannelElements.cc:9-19) */
static v4 lt_(v4 a, v4 b, v4 c) {
    double t = a.x * b.y * c.z + a.y * b.z * c.x + a.z * b.x * c.y - a.x * b.z * c.y - a.z * b.y * c.x - a.y * b.x * c.z;
    double x = -a.e * b.y * c.z - a.y * b.z * c.e - a.z * b.e * c.y + a.e * b.z * c.y + a.z * b.y * c.e + a.y * b.e * c.z;
    double y = -a.x * b.e * c.z - a.e * b.z * c.x - a.z * b.x * c.e + a.x * b.z * c.e + a.z * b.e * c.x + a.e * b.x * c.z;
    double z = -a.x * b.y * c.e - a.y * b.e * c.x - a.e * b.x * c.y + a.x * b.e * c.y + a.e * b.y * c.x + a.y * b.x * c.e;
    v4 r = {t, -x, -y, -z};
    return r;
}
static double get_(v4 a, int i) { return i == 0 ? a.e : i == 1 ? a.x : i == 2 ? a.y : a.z; }
static void put_(v4 *a, int i, double v) { if (i == 0) a->e = v; else if (i == 1) a->x = v; else if (i == 2) a->y = v; else a->z = v; }
/* m_t of Poincare(v1, v2) (Poincare.cc:10-34) */
static v4 rot_pt(v4 v1, v4 v2) {
    double n2 = sqrt(p2_(v2)), n1 = sqrt(p2_(v1));
    v4 b = {0., v2.x / n2, v2.y / n2, v2.z / n2};
    v4 l = {0., v1.x / n1, v1.y / n1, v1.z / n1};
    v4 t = vadd(b, vmul(l, mdot(l, b)));
    double mt = p2_(t);
    if (mt != 0.) t = vmul(t, 1. / sqrt(mt));
    int q[3] = {1, 2, 3};
    double ml[4] = {0., fabs(l.x), fabs(l.y), fabs(l.z)};
    int s;
    if (ml[q[2]] > ml[q[1]]) { s = q[1]; q[1] = q[2]; q[2] = s; }
    if (ml[q[1]] > ml[q[0]]) { s = q[0]; q[0] = q[1]; q[1] = s; }
    if (ml[q[2]] > ml[q[1]]) { s = q[1]; q[1] = q[2]; q[2] = s; }
    double tdp = get_(t, q[1]) * get_(l, q[1]) + get_(t, q[2]) * get_(l, q[2]);
    if (tdp != 0.) put_(&t, q[0], -tdp / get_(l, q[0]));
    if (p2_(t) == 0.) put_(&t, q[1], 1.);
    return t;
}
/* Boost / BoostBack (Poincare.cc:36-50) */
static v4 boost_(v4 l, double rsq, v4 v, double sgn) {
    double lv = l.x * v.x + l.y * v.y + l.z * v.z;
    double v0 = (l.e * v.e + sgn * lv) / rsq;
    double c1 = (v.e + v0) / (rsq + l.e);
    v4 r = {v0, v.x + sgn * (l.x * c1), v.y + sgn * (l.y * c1), v.z + sgn * (l.z * c1)};
    return r;
}
/* SmallOMCT (FourVector.cc:57-65) */
static double omct(v4 a, v4 v) {
    double mag = sqrt(p2_(a) * p2_(v)), pq = dot3_(a, v);
    double ct = dmin_(dmax_(pq / mag, -1.), 1.);
    if (ct < 0.) return 1. - ct;
    double cx = a.y * v.z - a.z * v.y, cy = a.z * v.x - a.x * v.z, cz = a.x * v.y - a.y * v.x;
    double st = sqrt(cx * cx + cy * cy + cz * cz) / mag;
    double st2 = st / (2. * sqrt((ct + 1) / 2.));
    return 2. * st2 * st2;
}
/* SChannelMomenta (ChannelElements.cc:87-111) with ctmin=-1, ctmax=1, xref=(1,1,0,0) */
static void sch_mom(v4 p, double s1, double s2, v4 *p1, v4 *p2, double r1, double r2) {
    double s = m2_(p), rs = sqrt(fabs(s));
    double e1 = (s + s1 - s2) / rs / 2., m1 = sqrt(e1 * e1 - s1);
    double ct = -1. + 2. * r1, st = sqrt(1. - ct * ct), ph = 2. * PI * r2;
    v4 xref = {1., 1., 0., 0.}, zax = {1., 0., 0., 1.};
    v4 pl = p2_(p) != 0. ? p : zax;
    double rsq = sqrt(m2_(p));
    v4 np = rot_pt(pl, xref);
    v4 lp = lt_(pl, xref, np);
    lp = vmul(lp, 1.0 / sqrt(fabs(m2_(lp))));
    double pp = sqrt(p2_(pl)), mc = m1 * ct;
    v4 q = {e1, pl.x * mc / pp, pl.y * mc / pp, pl.z * mc / pp};
    q = vadd(q, vmul(vadd(vmul(lp, cos(ph)), vmul(np, sin(ph))), m1 * st));
    q = boost_(p, rsq, q, +1.);
    *p1 = q;
    *p2 = vsub(p, q);
}
/* SChannelWeight (ChannelElements.cc:113-135) */
static double sch_wgt(v4 p1, v4 p2, double *r1, double *r2) {
    v4 p = vadd(p1, p2), xref = {1., 1., 0., 0.}, zax = {1., 0., 0., 1.};
    v4 pl = p2_(p) != 0. ? p : zax;
    double rsq = sqrt(m2_(p));
    v4 np = rot_pt(pl, xref);
    v4 lp = lt_(pl, xref, np);
    lp = vmul(lp, 1.0 / sqrt(fabs(m2_(lp))));
    v4 h = boost_(p, rsq, p1, -1.);
    double ct = dot3_(h, pl) / sqrt(p2_(h) * p2_(pl));
    double cp = -mdot(lp, p1), sp = -mdot(np, p1), nn = sqrt(cp * cp + sp * sp);
    cp /= nn;
    sp /= nn;
    *r1 = (ct + 1.) / 2.;
    *r2 = atan2(sp, cp) / (2. * PI);
    if (*r2 < 0.) *r2 += 1.;
    double w = 1.;
    double s1 = dmax_(m2_(p1), 0.), s2 = dmax_(m2_(p2), 0.), s = m2_(p);
    if (s1 == 0. && s2 == 0.) s = p1.e * p2.e * omct(p1, p2);
    w *= sqlam(s, s1, s2) / (8. * PI);
    return w;
}

/* --------------------------------------------------------------- FSMapper */
#define NSLOT (2 * CHILI_MAX_EXT)
typedef struct {
    int n_ext, ndims, n_slots;
    double sqrts, ptmax;
    double m2ext[NSLOT];
    int n_info, info_slot[CHILI_MAX_EXT];
    double info_ptmin[CHILI_MAX_EXT], info_etamax[CHILI_MAX_EXT];
    int n_dec, dp[CHILI_MAX_EXT], da[CHILI_MAX_EXT], db[CHILI_MAX_EXT], dml[CHILI_MAX_EXT];
    double dm[CHILI_MAX_EXT], dw[CHILI_MAX_EXT], dsmin2[CHILI_MAX_EXT], dcut[CHILI_MAX_EXT], dsmax[CHILI_MAX_EXT];
    int n_sd, sab[CHILI_MAX_EXT], sa[CHILI_MAX_EXT], sb[CHILI_MAX_EXT];
} chan_t;

static int cmp_info(const chili_particle_info *a, const chili_particle_info *b) { /* ChannelNode.cc:293-301 */
    if (a->idx != b->idx) return a->idx < b->idx ? -1 : 1;
    if (a->mass != b->mass) return a->mass < b->mass ? -1 : 1;
    if (a->width != b->width) return a->width < b->width ? -1 : 1;
    return 0;
}
static int cmp_decay(const void *a, const void *b) {
    return cmp_info(&((const chili_decay *)a)->parent, &((const chili_decay *)b)->parent);
}
static int lookup_iv(const chili_idx_value *t, int n, uint32_t idx, double *v) {
    for (int i = 0; i < n; ++i) if (t[i].idx == idx) { *v = t[i].value; return 1; }
    return 0;
}
static int is_pow2(uint32_t v) { return (v & (v - 1)) == 0; }

typedef struct { const chili_decay *d; int n; } decmap;
static const chili_decay *find_decay(const decmap *m, const chili_particle_info *key) {
    for (int i = 0; i < m->n; ++i) if (cmp_info(&m->d[i].parent, key) == 0) return &m->d[i];
    return NULL;
}
static int schedule(chan_t *c, const decmap *m, const int *slot, const chili_particle_info *ab) {
    const chili_decay *d = find_decay(m, ab);
    if (!d || c->n_sd >= CHILI_MAX_EXT) return 0;
    c->sab[c->n_sd] = slot[ab->idx];
    c->sa[c->n_sd] = slot[d->child1.idx];
    c->sb[c->n_sd] = slot[d->child2.idx];
    c->n_sd++;
    if (!is_pow2(d->child1.idx) && !schedule(c, m, slot, &d->child1)) return 0;
    if (!is_pow2(d->child2.idx) && !schedule(c, m, slot, &d->child2)) return 0;
    return 1;
}

/* FSMapper constructor (Channel.hh:18-30) plus the decay order of the
 * std::map DecayMap; returns 0 on an inconsistent description. */
static int build_chan(chan_t *c, const chili_channel_desc *d, const chili_cuts *cu, double sqrts, int n_ext) {
    memset(c, 0, sizeof(*c));
    int nout = n_ext - 2;
    c->n_ext = n_ext;
    c->ndims = 3 * nout - 4 + 2; /* Channel.hh:33 */
    c->sqrts = sqrts;
    c->ptmax = sqrts / 2.0;
    int slot[1 << CHILI_MAX_EXT];
    for (int i = 0; i < (1 << CHILI_MAX_EXT); ++i) slot[i] = -1;
    for (int i = 0; i < n_ext; ++i) slot[1u << i] = i;
    for (int i = 0; i < nout; ++i) c->m2ext[i + 2] = cu->sexternal[i];
    int ns = n_ext;
    if (d->n_decays > CHILI_MAX_EXT || d->n_info < 1 || d->n_info > nout) return 0;
    chili_decay *dec = malloc(sizeof(chili_decay) * (d->n_decays > 0 ? d->n_decays : 1));
    if (d->n_decays) memcpy(dec, d->decays, sizeof(chili_decay) * d->n_decays);
    qsort(dec, d->n_decays, sizeof(chili_decay), cmp_decay);
    decmap m = {dec, d->n_decays};
    for (int k = 0; k < d->n_decays; ++k) {
        uint32_t p = dec[k].parent.idx;
        if (slot[p] < 0) slot[p] = ns++;
    }
    c->n_slots = ns;
    for (int k = 0; k < d->n_decays; ++k) {
        const chili_decay *q = &dec[k];
        double pt1, pt2, dr = 0, cut = 0;
        if (!lookup_iv(cu->ptmin, cu->n_ptmin, q->child1.idx, &pt1) || !lookup_iv(cu->ptmin, cu->n_ptmin, q->child2.idx, &pt2)) {
            free(dec);
            return 0;
        }
        for (int i = 0; i < cu->n_deltaR; ++i)
            if (cu->deltaR[i].pid1 == q->child1.pid && cu->deltaR[i].pid2 == q->child2.pid) dr = cu->deltaR[i].value;
        lookup_iv(cu->smin, cu->n_smin, q->child1.idx | q->child2.idx, &cut);
        double smax = sqrts; /* SMax (Cuts.hh:21-29) */
        for (int i = 0; i < cu->n_sexternal; ++i)
            if (!(q->parent.idx & (1u << (i + 2)))) smax -= sqrt(cu->sexternal[i]);
        c->dp[k] = slot[q->parent.idx];
        c->da[k] = slot[q->child1.idx];
        c->db[k] = slot[q->child2.idx];
        if (c->da[k] < 0 || c->db[k] < 0) { free(dec); return 0; }
        c->dml[k] = (fabs(q->parent.mass) < 1e-16 || q->parent.width < 1e-16);
        c->dm[k] = q->parent.mass;
        c->dw[k] = q->parent.width;
        c->dsmin2[k] = pt1 * pt2 * 2 / PI / PI * pow(dr, 2); /* Channel.cc:150 */
        c->dcut[k] = cut;
        c->dsmax[k] = smax * smax;
    }
    c->n_dec = d->n_decays;
    c->n_info = d->n_info;
    for (int i = 0; i < d->n_info; ++i) {
        double pt, eta;
        uint32_t idx = d->info[i].idx;
        if (idx >= (1u << CHILI_MAX_EXT) || slot[idx] < 0 || !lookup_iv(cu->ptmin, cu->n_ptmin, idx, &pt) ||
            !lookup_iv(cu->etamax, cu->n_etamax, idx, &eta)) {
            free(dec);
            return 0;
        }
        c->info_slot[i] = slot[idx];
        c->info_ptmin[i] = pt != 0 ? pt : 1;
        c->info_etamax[i] = eta;
    }
    for (int i = 0; i < d->n_info; ++i)
        if (!is_pow2(d->info[i].idx) && !schedule(c, &m, slot, &d->info[i])) { free(dec); return 0; }
    free(dec);
    return c->n_dec + 3 * (c->n_info - 1) + 1 + 2 * c->n_sd == c->ndims;
}

/* GeneratePoint (Channel.cc:22-38): GenDecays :63-81, GenTChan :115-158,
 * GenSChan/DecayParts :204-245. */
static void fs_gen(const chan_t *c, const double *x, v4 *mom) {
    double m2[NSLOT];
    memcpy(m2, c->m2ext, sizeof(m2));
    int ir = 0;
    for (int k = 0; k < c->n_dec; ++k) {
        double r = sqrt(m2[c->da[k]]) + sqrt(m2[c->db[k]]);
        double smin = dmax_(dmax_(r * r, c->dsmin2[k]), c->dcut[k]);
        double u = x[ir++];
        m2[c->dp[k]] = c->dml[k] ? ml_mom(0.99, smin, c->dsmax[k], u) : bw_mom(c->dm[k], c->dw[k], smin, c->dsmax[k], u);
    }
    v4 ps = {0, 0, 0, 0};
    double S = c->sqrts, PM = c->ptmax;
    for (int i = 0; i < c->n_info - 1; ++i) {
        double pmn = c->info_ptmin[i], ran = x[ir++];
        double pt = 2 * pmn * PM * ran / (2 * pmn + PM * (1 - ran));
        double em = S / 2 / pt;
        em = log(em + sqrt(em * em - 1));
        em = dmin_(em, c->info_etamax[i]);
        double y = em * (2 * x[ir++] - 1), sh = sinh(y), ch = sqrt(1 + sh * sh), ph = 2 * PI * x[ir++];
        int s = c->info_slot[i];
        double mt = sqrt(pt * pt + m2[s]);
        v4 q = {mt * ch, pt * cos(ph), pt * sin(ph), mt * sh};
        mom[s] = q;
        ps = vadd(ps, q);
    }
    {
        int s = c->info_slot[c->n_info - 1];
        double mj2 = m2_(ps), yj = rap_(ps), ptj2 = pt2_(ps);
        double qt = sqrt(m2[s] + ptj2), mt = sqrt(mj2 + ptj2);
        double ymin = -log(S / qt * (1 - mt / S * exp(-yj)));
        double ymax = log(S / qt * (1 - mt / S * exp(yj)));
        double yv = ymin + x[ir++] * (ymax - ymin), sh = sinh(yv), ch = sqrt(1 + sh * sh);
        v4 q = {qt * ch, -ps.x, -ps.y, qt * sh};
        mom[s] = q;
        v4 t = vadd(q, ps);
        double pp = t.e + t.z, pm = t.e - t.z;
        v4 a = {-pp / 2, 0, 0, -pp / 2}, b = {-pm / 2, 0, 0, pm / 2};
        mom[0] = a;
        mom[1] = b;
    }
    for (int k = 0; k < c->n_sd; ++k) {
        double r1 = x[ir++], r2 = x[ir++];
        sch_mom(mom[c->sab[k]], m2[c->sa[k]], m2[c->sb[k]], &mom[c->sa[k]], &mom[c->sb[k]], r1, r2);
    }
}

/* GenerateWeight (Channel.cc:40-61): WgtDecays :83-113, WgtTChan :160-202
 * (returns 0 without its last uniform when ymin/ymax are NaN), WgtSChan
 * :222-256. */
static double fs_wgt(const chan_t *c, v4 *mom, double *x) {
    for (int k = 0; k < c->n_dec; ++k) mom[c->dp[k]] = vadd(mom[c->da[k]], mom[c->db[k]]);
    int ir = 0;
    double wd = 1;
    for (int k = 0; k < c->n_dec; ++k) {
        double r = sqrt(fabs(m2_(mom[c->da[k]]))) + sqrt(fabs(m2_(mom[c->db[k]])));
        double smin = dmax_(dmax_(r * r, c->dsmin2[k]), c->dcut[k]), s = m2_(mom[c->dp[k]]), u;
        wd *= c->dml[k] ? ml_wgt(0.99, smin, c->dsmax[k], s, &u) : bw_wgt(c->dm[k], c->dw[k], smin, c->dsmax[k], s, &u);
        x[ir++] = u;
        wd /= (2 * PI);
    }
    double S = c->sqrts, PM = c->ptmax, wt = 2 * PI;
    const double inv = 1.0 / (16 * pow(PI, 3));
    v4 ps = {0, 0, 0, 0};
    for (int i = 0; i < c->n_info - 1; ++i) {
        double pmn = c->info_ptmin[i];
        v4 q = mom[c->info_slot[i]];
        wt *= inv;
        double pt = sqrt(pt2_(q)), f2 = 2 * pmn + pt;
        wt *= pt * PM / 2 / pmn / (2 * pmn + PM) * (f2 * f2);
        x[ir++] = pt * (PM + 2 * pmn) / (PM * (pt + 2 * pmn));
        double em = S / 2 / pt;
        em = log(em + sqrt(em * em - 1));
        em = isnan(em) ? 99 : em;
        em = dmin_(em, c->info_etamax[i]);
        wt *= 2 * em * 2 * PI;
        x[ir++] = (rap_(q) / em + 1) / 2;
        x[ir++] = phi_(q) / 2 / PI;
        ps = vadd(ps, q);
    }
    {
        v4 q = mom[c->info_slot[c->n_info - 1]];
        double mj2 = m2_(ps), yj = rap_(ps), ptj2 = pt2_(ps), m2 = m2_(q);
        double qt = sqrt(m2 + ptj2), mt = sqrt(mj2 + ptj2), yv = rap_(q);
        double ymin = -log(S / qt * (1 - mt / S * exp(-yj)));
        double ymax = log(S / qt * (1 - mt / S * exp(yj)));
        double dely = ymax - ymin;
        if (isnan(ymax) || isnan(ymin)) wt = 0;
        else {
            wt *= dely / S / S;
            x[ir++] = (yv - ymin) / dely;
        }
    }
    double ws = 1;
    for (int k = 0; k < c->n_sd; ++k) {
        double r1, r2;
        ws *= sch_wgt(mom[c->sa[k]], mom[c->sb[k]], &r1, &r2);
        x[ir++] = r1;
        x[ir++] = r2;
    }
    return wd * wt * ws;
}

/* ---------------------------------------------------------- multichannel */
typedef struct {
    int nch, n_ext, ndims, bins;
    chan_t *ch;
    double *grids; /* nch * ndims * (bins+1) */
    double *alpha, *best, min_diff;
    int best_set;
    chili_multichannel_params prm;
    int fkind, pre;
    double fp[CHILI_MAX_INTEGRAND_PARAMS];
    double cut[4]; /* CHILI_PRE_CUTS: sqrts, ptmin, etamax, delta_r */
    int defer;     /* collect the training data, leave Train to the caller */
    int fixed;     /* fixed budget: rejected and NaN points are calls of value 0, no retry */
    double *hist, *atrain;
} mc_t;

/* CHILI_PRE_CUTS (include/chili_gpu.h): physical region and cuts; a
 * PreProcess callback of this harness, not a reference step. */
static int pass_cuts(const mc_t *m, const v4 *q) {
    const double half = 0.5 * m->cut[0] * (1.0 + 1e-12);
    if (!(-q[0].e <= half) || !(-q[1].e <= half)) return 0;
    const double pt2min = m->cut[1] * m->cut[1], etamax = m->cut[2], dr2 = m->cut[3] * m->cut[3];
    double eta[CHILI_MAX_EXT], phi[CHILI_MAX_EXT];
    for (int i = 2; i < m->n_ext; ++i) {
        const double pt2 = q[i].x * q[i].x + q[i].y * q[i].y;
        if (!(pt2 >= pt2min) || !(pt2 > 0)) return 0;
        eta[i] = asinh(q[i].z / sqrt(pt2));
        if (!(fabs(eta[i]) <= etamax)) return 0;
        phi[i] = atan2(q[i].y, q[i].x);
    }
    for (int i = 2; i < m->n_ext; ++i)
        for (int j = i + 1; j < m->n_ext; ++j) {
            double dphi = fabs(phi[i] - phi[j]);
            if (dphi > 3.14159265358979323846) dphi = 2.0 * 3.14159265358979323846 - dphi;
            const double deta = eta[i] - eta[j];
            if (!(deta * deta + dphi * dphi >= dr2)) return 0;
        }
    return 1;
}

/* PreProcess of the harness: 1 = accepted. */
static int preprocess_ok(const mc_t *m, const v4 *q) {
    if (m->pre == CHILI_PRE_FINITE) return !isnan(q[0].e);
    if (m->pre == CHILI_PRE_CUTS) return pass_cuts(m, q);
    return 1;
}

/* std::discrete_distribution (libstdc++ _M_initialize / operator()) as used
 * by Random::SelectIndex (Random.hh:43-45). */
static int select1(const double *a, int n, double v) {
    if (n < 2) return 0;
    double sum = 0, cp[CHILI_MAX_CHANNELS];
    for (int i = 0; i < n; ++i) sum += a[i];
    double acc = 0;
    for (int i = 0; i < n; ++i) {
        double p = a[i] / sum;
        acc = i == 0 ? p : acc + p;
        cp[i] = acc;
    }
    cp[n - 1] = 1.0;
    int first = 0, len = n;
    while (len > 0) {
        int half = len >> 1, mid = first + half;
        if (cp[mid] < v) { first = mid + 1; len = len - half - 1; }
        else len = half;
    }
    return first < n ? first : n - 1;
}
void orc_select(const double *a, int n, const double *v, int64_t m, int32_t *out) {
    for (int64_t i = 0; i < m; ++i) out[i] = select1(a, n, v[i]);
}

void *orc_mc_create(const chili_channel_desc *d, int nch, const chili_cuts *cu, double sqrts, int n_ext, int bins,
                    const chili_multichannel_params *prm) {
    if (nch < 1 || nch > CHILI_MAX_CHANNELS || n_ext < 3 || n_ext > CHILI_MAX_EXT || bins < 2) return NULL;
    mc_t *m = calloc(1, sizeof(mc_t));
    m->nch = nch;
    m->n_ext = n_ext;
    m->ndims = 3 * (n_ext - 2) - 2;
    m->bins = bins;
    m->ch = calloc(nch, sizeof(chan_t));
    for (int c = 0; c < nch; ++c)
        if (!build_chan(&m->ch[c], &d[c], cu, sqrts, n_ext)) { free(m->ch); free(m); return NULL; }
    size_t gs = (size_t)m->ndims * (bins + 1);
    m->grids = malloc(sizeof(double) * gs * nch);
    for (int c = 0; c < nch; ++c)
        for (int dd = 0; dd < m->ndims; ++dd)
            for (int k = 0; k <= bins; ++k) m->grids[c * gs + dd * (bins + 1) + k] = (double)k / (double)bins;
    m->alpha = malloc(sizeof(double) * nch);
    m->best = malloc(sizeof(double) * nch);
    for (int c = 0; c < nch; ++c) { m->alpha[c] = 1.0 / (double)nch; m->best[c] = NAN; }
    m->min_diff = INFINITY;
    m->prm = *prm;
    m->hist = calloc((size_t)nch * m->ndims * bins, sizeof(double));
    m->atrain = calloc(nch, sizeof(double));
    m->fkind = CHILI_FUNC_UNIT;
    m->pre = CHILI_PRE_FINITE;
    return m;
}
void orc_mc_destroy(void *p) {
    mc_t *m = p;
    if (!m) return;
    free(m->ch); free(m->grids); free(m->alpha); free(m->best); free(m->hist); free(m->atrain); free(m);
}
int orc_mc_ndims(void *p) { return ((mc_t *)p)->ndims; }
void orc_mc_set_integrand(void *p, int kind, const double *fp, int np, int pre) {
    mc_t *m = p;
    m->fkind = kind;
    m->pre = pre;
    for (int i = 0; i < np && i < CHILI_MAX_INTEGRAND_PARAMS; ++i) m->fp[i] = fp[i];
}
void orc_mc_set_cuts(void *p, double sqrts, double ptmin, double etamax, double dr) {
    mc_t *m = p;
    m->pre = CHILI_PRE_CUTS;
    m->cut[0] = sqrts; m->cut[1] = ptmin; m->cut[2] = etamax; m->cut[3] = dr;
}
void orc_mc_set_grids(void *p, const double *e) {
    mc_t *m = p;
    memcpy(m->grids, e, sizeof(double) * m->nch * m->ndims * (m->bins + 1));
}
void orc_mc_get_grids(void *p, double *e) {
    mc_t *m = p;
    memcpy(e, m->grids, sizeof(double) * m->nch * m->ndims * (m->bins + 1));
}
void orc_mc_set_alpha(void *p, const double *a) { mc_t *m = p; memcpy(m->alpha, a, sizeof(double) * m->nch); }
void orc_mc_get_alpha(void *p, double *a, double *b, double *md) {
    mc_t *m = p;
    if (a) memcpy(a, m->alpha, sizeof(double) * m->nch);
    if (b) memcpy(b, m->best, sizeof(double) * m->nch);
    if (md) *md = m->min_diff;
}
void orc_fsm_generate(void *p, int c, const double *x, int64_t n, double *mom) {
    mc_t *m = p;
    for (int64_t i = 0; i < n; ++i) {
        v4 q[NSLOT];
        fs_gen(&m->ch[c], x + i * m->ndims, q);
        memcpy(mom + i * m->n_ext * 4, q, sizeof(double) * 4 * m->n_ext);
    }
}
void orc_fsm_weight(void *p, int c, const double *mom, int64_t n, double *xo, double *w) {
    mc_t *m = p;
    for (int64_t i = 0; i < n; ++i) {
        v4 q[NSLOT];
        double x[CHILI_MAX_DIMS] = {0};
        memcpy(q, mom + i * m->n_ext * 4, sizeof(double) * 4 * m->n_ext);
        w[i] = fs_wgt(&m->ch[c], q, x);
        if (xo) memcpy(xo + i * m->ndims, x, sizeof(double) * m->ndims);
    }
}

/* Integrand::GenerateWeight (Integrand.hh:112-123): one uniform buffer shared
 * by all channels and never cleared between them. */
static double combined(mc_t *m, const v4 *mom0, int ich, double *dens, double *xs) {
    double x[CHILI_MAX_DIMS] = {0}, acc = 0;
    v4 q[NSLOT];
    memcpy(q, mom0, sizeof(v4) * m->n_ext);
    size_t gs = (size_t)m->ndims * (m->bins + 1);
    for (int c = 0; c < m->nch; ++c) {
        dens[c] = fs_wgt(&m->ch[c], q, x);
        if (c == ich) memcpy(xs, x, sizeof(double) * m->ndims);
        double vw = am_weight1(m->grids + c * gs, m->ndims, m->bins, x);
        acc += m->alpha[c] / dens[c] / vw;
    }
    return 1.0 / acc;
}
void orc_mc_weight(void *p, const double *mom, const int32_t *ich, int64_t n, double *w, double *dens, double *xs) {
    mc_t *m = p;
    double d[CHILI_MAX_CHANNELS], x[CHILI_MAX_DIMS] = {0};
    for (int64_t i = 0; i < n; ++i) {
        w[i] = combined(m, (const v4 *)(mom + i * m->n_ext * 4), ich[i], d, x);
        if (dens) memcpy(dens + i * m->nch, d, sizeof(double) * m->nch);
        if (xs) memcpy(xs + i * m->ndims, x, sizeof(double) * m->ndims);
    }
}
static double eval_f(const mc_t *m, const v4 *mom) {
    if (m->fkind == CHILI_FUNC_PROPAGATOR) return propagator(m->fp, mom, m->n_ext, 0);
    if (m->fkind == CHILI_FUNC_PROPAGATOR_TOP2) return propagator(m->fp, mom, m->n_ext, 1);
    return 1.0;
}

/* MultiChannel::Train (MultiChannel.hh:182-194): Adapt (MultiChannel.cc:109-136)
 * from the alpha-training sums, Integrand::Train (Integrand.hh:97-104) from the
 * per-channel histograms, MaxDifference (MultiChannel.cc:138-154). In the
 * reference's MPI mode both inputs are the all-reduced sums of the ranks. */
static void mc_train(mc_t *m, const double *train, const double *hist) {
    int D = m->ndims, B = m->bins, nch = m->nch;
    size_t gs = (size_t)D * (B + 1);
    double nw[CHILI_MAX_CHANNELS], sw = 0, ns = 0;
    for (int i = 0; i < nch; ++i) { nw[i] = m->alpha[i] * pow(train[i], m->prm.beta); sw += nw[i]; }
    for (int i = 0; i < nch; ++i) {
        if (nw[i] == 0) continue;
        nw[i] /= sw;
        nw[i] = dmax_(nw[i], m->prm.min_alpha);
        ns += nw[i];
    }
    for (int i = 0; i < nch; ++i) m->alpha[i] = nw[i] / ns;
    for (int c = 0; c < nch; ++c) {
        const double *h = hist + (size_t)c * D * B;
        int nz = 0;
        for (int q = 0; q < D * B; ++q) nz |= h[q] != 0;
        if (nz) am_adapt1(m->grids + c * gs, D, B, m->prm.grid_alpha, h);
    }
    double mx = 0;
    for (int i = 0; i + 1 < nch; ++i)
        for (int j = i + 1; j < nch; ++j) mx = dmax_(mx, fabs(train[i] - train[j]));
    if (mx < m->min_diff) { memcpy(m->best, m->alpha, sizeof(double) * nch); m->min_diff = mx; }
}
void orc_mc_train(void *p, const double *hist, const double *atrain) { mc_train((mc_t *)p, atrain, hist); }
void orc_mc_set_defer(void *p, int defer) { ((mc_t *)p)->defer = defer; }
/* The batched integrands' semantics (not the reference's): every drawn point
 * is one of the ncalls calls, PreProcess rejections and NaN values included
 * as calls of value 0; MultiChannel.hh:219-236 otherwise. */
void orc_mc_set_fixed_budget(void *p, int on) { ((mc_t *)p)->fixed = on; }

/* MultiChannel::operator() (MultiChannel.hh:196-251) on given uniforms, with
 * Train (:182-194) = Adapt (MultiChannel.cc:109-136), Integrand::Train
 * (Integrand.hh:97-104) and MaxDifference (MultiChannel.cc:138-154). */
int orc_mc_iterate(void *p, const double *u, int64_t n_u, int guard, chili_stats *out, chili_mc_iter_info *info) {
    mc_t *m = p;
    int D = m->ndims, B = m->bins, nch = m->nch;
    size_t gs = (size_t)D * (B + 1);
    memset(m->hist, 0, sizeof(double) * nch * D * B);
    double *train = calloc(nch, sizeof(double));
    memset(info, 0, sizeof(*info));
    stats_t st;
    st_init(&st);
    int64_t k = 0;
    uint64_t ncalls = m->prm.ncalls;
    double dens[CHILI_MAX_CHANNELS];
    for (uint64_t i = 0; i < ncalls; ++i) {
        if (k >= n_u) { free(train); return CHILI_ERR_LIMIT; }
        const double *uk = u + k * (D + 1);
        ++k;
        double x[CHILI_MAX_DIMS], xs[CHILI_MAX_DIMS] = {0}, jac;
        memcpy(x, uk, sizeof(double) * D);
        int ich = select1(m->alpha, nch, uk[D]);
        v4 mom[NSLOT];
        if (am_map1(m->grids + ich * gs, D, B, x, &jac)) fs_gen(&m->ch[ich], x, mom);
        else for (int s = 0; s < m->n_ext; ++s) { v4 z = {NAN, NAN, NAN, NAN}; mom[s] = z; }
        if (!preprocess_ok(m, mom)) {
            if (!m->fixed) --i;
            st_add(&st, 0);
            info->rejected_pre++;
            continue;
        }
        double wgt = combined(m, mom, ich, dens, xs);
        double f = eval_f(m, mom);
        double val = wgt == 0 ? 0 : f * wgt;
        if (isnan(val)) { val = wgt = 0; if (!m->fixed) --i; info->rejected_nan++; }
        if (m->prm.should_optimize) {
            double v2 = val * val;
            double *h = m->hist + (size_t)ich * D * B;
            const double *g = m->grids + ich * gs;
            for (int j = 0; j < D; ++j) {
                int s = j * B + find_bin(g + j * (B + 1), B, xs[j]);
                if (s >= 0) h[s] += v2; /* dim 0, FindBin SIZE_MAX: would write before the histogram */
            }
            for (int j = 0; j < nch; ++j) {
                double t = v2 * wgt / dens[j];
                if (guard && !isfinite(t)) { info->nonfinite_alpha_terms += 1; continue; }
                train[j] += t;
            }
        }
        if (val > info->weight_max) info->weight_max = val;
        st_add(&st, val);
    }
    info->points_tried = (uint64_t)k;
    info->points_accepted = ncalls;
    info->points_weighted = ncalls + info->rejected_nan;
    memcpy(m->atrain, train, sizeof(double) * nch);
    if (m->prm.should_optimize && !m->defer) mc_train(m, train, m->hist);
    free(train);
    st_out(&st, out);
    return 0;
}
/* The value of each point of MultiChannel::operator() (MultiChannel.hh:
 * 214-233) without retries: uniforms u[n][D+1] -> channel, momenta, value
 * f * w (0 for a PreProcess rejection or a NaN value); the input of the
 * unweighting stage.  mom (n * n_ext * 4) and ich may be NULL. */
void orc_mc_point_values(void *p, const double *u, int64_t n, double *val, int32_t *ich_out, double *mom_out) {
    mc_t *m = p;
    int D = m->ndims, B = m->bins;
    size_t gs = (size_t)D * (B + 1);
    double dens[CHILI_MAX_CHANNELS];
    for (int64_t i = 0; i < n; ++i) {
        const double *uk = u + i * (D + 1);
        double x[CHILI_MAX_DIMS], xs[CHILI_MAX_DIMS] = {0}, jac;
        memcpy(x, uk, sizeof(double) * D);
        int ich = select1(m->alpha, m->nch, uk[D]);
        v4 mom[NSLOT];
        if (am_map1(m->grids + ich * gs, D, B, x, &jac)) fs_gen(&m->ch[ich], x, mom);
        else for (int s = 0; s < m->n_ext; ++s) { v4 z = {NAN, NAN, NAN, NAN}; mom[s] = z; }
        double v = 0;
        if (preprocess_ok(m, mom)) {
            double wgt = combined(m, mom, ich, dens, xs);
            double f = eval_f(m, mom);
            v = wgt == 0 ? 0 : f * wgt;
            if (isnan(v)) v = 0;
        }
        val[i] = v;
        if (ich_out) ich_out[i] = ich;
        if (mom_out) memcpy(mom_out + i * m->n_ext * 4, mom, sizeof(double) * 4 * m->n_ext);
    }
}
void orc_mc_get_training(void *p, double *h, double *a) {
    mc_t *m = p;
    if (h) memcpy(h, m->hist, sizeof(double) * m->nch * m->ndims * m->bins);
    if (a) memcpy(a, m->atrain, sizeof(double) * m->nch);
}

/* Interface::Evaluate (nanobind.hh:23-50) */
void orc_evaluate_batch(void *p, int c, const double *u, int64_t n, double *out) {
    mc_t *m = p;
    for (int64_t i = 0; i < n; ++i) {
        double x[CHILI_MAX_DIMS];
        memcpy(x, u + i * m->ndims, sizeof(double) * m->ndims);
        v4 q[NSLOT];
        fs_gen(&m->ch[c], x, q);
        if (!preprocess_ok(m, q)) { out[i] = 0; continue; }
        double w = fs_wgt(&m->ch[c], q, x);
        out[i] = w == 0 ? 0 : eval_f(m, q) * w;
    }
}

/* ------------------------------------------------------------ plain VEGAS */
/* Vegas::operator() (Vegas.cc:18-52) on given uniforms; edges adapted in
 * place when adapt != 0. */
void orc_vegas_iterate(int dims, int bins, double *edges, double alpha, int adapt, const double *fp, int np,
                       int64_t n, const double *u, chili_stats *out, double *train_out) {
    (void)np;
    double *train = calloc((size_t)dims * bins, sizeof(double));
    stats_t st;
    st_init(&st);
    for (int64_t i = 0; i < n; ++i) {
        double x[CHILI_MAX_DIMS], jac, val;
        memcpy(x, u + i * dims, sizeof(double) * dims);
        if (am_map1(edges, dims, bins, x, &jac)) val = camel(fp, x, dims) * jac;
        else val = NAN;
        double v2 = val * val;
        st_add(&st, val);
        for (int j = 0; j < dims; ++j) {
            int s = j * bins + find_bin(edges + j * (bins + 1), bins, x[j]);
            if (s >= 0) train[s] += v2;
        }
    }
    if (train_out) memcpy(train_out, train, sizeof(double) * dims * bins);
    if (adapt) am_adapt1(edges, dims, bins, alpha, train);
    free(train);
    st_out(&st, out);
}
