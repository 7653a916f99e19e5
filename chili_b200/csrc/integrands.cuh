// integrands.cuh -- built-in device integrands, selected by id.
//
// In the reference an integrand is a std::function (Vegas.hh:27-28,
// Integrand.hh:41-47) and cannot cross to the device; the workloads' own
// integrands are compiled in and chosen by chili_integrand_kind.
#pragma once

#include "chili_gpu.h"
#include "common.cuh"

namespace chili_dev {

struct IntegrandDesc {
    int32_t kind;
    int32_t nparams;
    int32_t pre;  // chili_preprocess_kind
    int32_t n_ext;  // external legs (CHILI_PRE_CUTS)
    double p[CHILI_MAX_INTEGRAND_PARAMS];
    double cut[4];  // CHILI_PRE_CUTS: sqrts, ptmin, etamax, delta_r
};

// f(x) = N [exp(-|x-a|^2/s^2) + exp(-|x-b|^2/s^2)]; params {s, N, a[D], b[D]}.
__device__ __forceinline__ double camel(const IntegrandDesc *__restrict__ f, const double *x, int dims) {
    const double s = f->p[0], norm = f->p[1];
    double d1 = 0, d2 = 0;
    for (int i = 0; i < dims; ++i) {
        double t = x[i] - f->p[2 + i];
        d1 += t * t;
        t = x[i] - f->p[2 + dims + i];
        d2 += t * t;
    }
    const double s2 = s * s;
    return norm * (exp(-d1 / s2) + exp(-d2 / s2));
}

// Pair Breit-Wigner sum (or product of the two largest) times the t-channel
// factors over the outgoing legs; params {M, G, m}.
__device__ __forceinline__ double propagator(const IntegrandDesc *__restrict__ f, const V4 *mom, int n_ext,
                                             bool top2) {
    const double m = f->p[0], g = f->p[1], mt = f->p[2];
    const double m2 = m * m, mw2 = m * m * g * g, mt2 = mt * mt;
    double sum = 0, big1 = 0, big2 = 0;
    for (int i = 2; i < n_ext; ++i) {
        for (int j = i + 1; j < n_ext; ++j) {
            const double d = mass2(mom[i] + mom[j]) - m2;
            const double bw = 1.0 / (d * d + mw2);
            sum += bw;
            if (bw > big1) {
                big2 = big1;
                big1 = bw;
            } else if (bw > big2) {
                big2 = bw;
            }
        }
    }
    double tprod = 1;
    for (int j = 2; j < n_ext; ++j) tprod *= 1.0 / (fabs(mass2(mom[0] + mom[j])) + mt2);
    return (top2 ? big1 * big2 : sum) * tprod;
}

__device__ __forceinline__ double eval_momenta(const IntegrandDesc *__restrict__ f, const V4 *mom, int n_ext) {
    switch (f->kind) {
    case CHILI_FUNC_PROPAGATOR: return propagator(f, mom, n_ext, false);
    case CHILI_FUNC_PROPAGATOR_TOP2: return propagator(f, mom, n_ext, true);
    default: return 1.0;
    }
}

// The physical region and the cuts of CHILI_PRE_CUTS (include/chili_gpu.h).
// NaN momenta fail every comparison.
__device__ __forceinline__ bool pass_cuts(const IntegrandDesc *__restrict__ f, const V4 *mom) {
    const double half = 0.5 * f->cut[0] * (1.0 + 1e-12);
    if (!(-mom[0].e <= half) || !(-mom[1].e <= half)) return false;
    const double pt2min = f->cut[1] * f->cut[1], etamax = f->cut[2], dr2 = f->cut[3] * f->cut[3];
    const int ne = f->n_ext;
    double eta[CHILI_MAX_EXT], phi[CHILI_MAX_EXT];
    for (int i = 2; i < ne; ++i) {
        const double pt2 = mom[i].x * mom[i].x + mom[i].y * mom[i].y;
        if (!(pt2 >= pt2min) || !(pt2 > 0)) return false;
        eta[i] = asinh(mom[i].z / sqrt(pt2));
        if (!(fabs(eta[i]) <= etamax)) return false;
        phi[i] = atan2(mom[i].y, mom[i].x);
    }
    for (int i = 2; i < ne; ++i)
        for (int j = i + 1; j < ne; ++j) {
            double dphi = fabs(phi[i] - phi[j]);
            if (dphi > kPi) dphi = 2.0 * kPi - dphi;
            const double deta = eta[i] - eta[j];
            if (!(deta * deta + dphi * dphi >= dr2)) return false;
        }
    return true;
}

// PreProcess (MultiChannel.hh:219-223); CHILI_PRE_FINITE follows the first
// check of src/example.cc:26-29.
__device__ __forceinline__ bool preprocess(const IntegrandDesc *__restrict__ f, const V4 *mom) {
    if (f->pre == CHILI_PRE_FINITE) return !isnan(mom[0].e);
    if (f->pre == CHILI_PRE_CUTS) return pass_cuts(f, mom);
    return true;
}

}  // namespace chili_dev
