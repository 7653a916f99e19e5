// fsmapper.cuh -- device FSMapper: uniforms -> FP64 four-momenta and the
// inverse (momenta -> uniforms, phase-space weight) of one flattened channel.
//
// Each function restates the reference step it cites (paths inside the Chili
// project) in device code; the operation order follows the reference so that
// results agree with its CPU build to rounding.
#pragma once

#include "channel_program.h"
#include "common.cuh"
#include "grid.cuh"

namespace chili_dev {

// ------------------------------------------------- channel elements
// SqLam (ChannelElements.cc:21-25)
__device__ __forceinline__ double sq_lambda(double s, double s1, double s2) {
    const double a = s - s1 - s2;
    const double arg = a * a - 4. * s1 * s2;
    if (arg > 0.) return sqrt(arg) / s;
    return 0.;
}

// PeakedDist / PeakedWeight with a = 0, k = 1 (ChannelElements.cc:27-50), as
// used by the massless propagator (:52-62): s^-cn sampling on [cxm, cxp].
__device__ __forceinline__ double massless_prop_momenta(double cn, double cxm, double cxp, double ran) {
    const double ce = 1. - cn;
    if (ce != 0.) return pow(ran * pow(cxp, ce) + (1. - ran) * pow(cxm, ce), 1 / ce);
    return cxm * pow(cxp / cxm, ran);
}
__device__ __forceinline__ double massless_prop_weight(double cn, double cxm, double cxp, double s,
                                                       double &ran) {
    const double ce = 1. - cn;
    double w;
    if (ce != 0.) {
        const double amin = pow(cxm, ce);
        w = pow(cxp, ce) - amin;
        ran = (pow(s, ce) - amin) / w;
        w /= ce;
    } else {
        const double amin = cxm;
        w = log(cxp / amin);
        ran = log(s / amin) / w;
    }
    return w / pow(s, -cn);
}

// The same weights with the (smin, smax)-only terms supplied: t1, t2 are
// pow(cxm, ce), pow(cxp, ce) (massless) or atan((smin-m2)/mw),
// atan((smax-m2)/mw) (massive), evaluated by the same functions, so the
// results are identical to the functions above.
__device__ __forceinline__ double massless_prop_weight_c(double cn, double t_min, double t_max, double s,
                                                         double &ran) {
    const double ce = 1. - cn;
    const double amin = t_min;
    double w = t_max - amin;
    ran = (pow(s, ce) - amin) / w;
    w /= ce;
    return w / pow(s, -cn);
}
__device__ __forceinline__ double massive_prop_weight_c(double m, double g, double ymax, double ymin, double s,
                                                        double &ran) {
    const double m2 = m * m, mw = m * g;
    const double y = atan((s - m2) / mw);
    ran = (y - ymin) / (ymax - ymin);
    double w = mw / ((s - m2) * (s - m2) + mw * mw);
    w = (ymin - ymax) / w;
    return w;
}

// Breit-Wigner propagator (ChannelElements.cc:64-85).
__device__ __forceinline__ double massive_prop_momenta(double m, double g, double smin, double smax,
                                                       double ran) {
    const double m2 = m * m, mw = m * g;
    const double ymax = atan((smin - m2) / mw), ymin = atan((smax - m2) / mw);
    return m2 + mw * tan(ymin + ran * (ymax - ymin));
}
__device__ __forceinline__ double massive_prop_weight(double m, double g, double smin, double smax,
                                                      double s, double &ran) {
    const double m2 = m * m, mw = m * g;
    const double ymax = atan((smin - m2) / mw), ymin = atan((smax - m2) / mw);
    const double y = atan((s - m2) / mw);
    ran = (y - ymin) / (ymax - ymin);
    double w = mw / ((s - m2) * (s - m2) + mw * mw);
    w = (ymin - ymax) / w;
    return w;
}

// LT: the 4-d cross product (ChannelElements.cc:9-19).
__device__ __forceinline__ V4 lorentz_cross(V4 a, V4 b, V4 c) {
    const double t = a.x * b.y * c.z + a.y * b.z * c.x + a.z * b.x * c.y - a.x * b.z * c.y -
                     a.z * b.y * c.x - a.y * b.x * c.z;
    const double x = -a.e * b.y * c.z - a.y * b.z * c.e - a.z * b.e * c.y + a.e * b.z * c.y +
                     a.z * b.y * c.e + a.y * b.e * c.z;
    const double y = -a.x * b.e * c.z - a.e * b.z * c.x - a.z * b.x * c.e + a.x * b.z * c.e +
                     a.z * b.e * c.x + a.e * b.x * c.z;
    const double z = -a.x * b.y * c.e - a.y * b.e * c.x - a.e * b.x * c.y + a.x * b.e * c.y +
                     a.e * b.y * c.x + a.y * b.x * c.e;
    return V4{t, -x, -y, -z};
}

// The transverse axis m_t of the rotation Poincare(v1, v2) (Poincare.cc:10-34).
__device__ __forceinline__ V4 rotation_axis(V4 v1, V4 v2) {
    const double pv2 = sqrt(p2(v2));
    const V4 b{0., v2.x / pv2, v2.y / pv2, v2.z / pv2};
    const double pv1 = sqrt(p2(v1));
    const V4 l{0., v1.x / pv1, v1.y / pv1, v1.z / pv1};
    V4 t = b + scale(l, dot4(l, b));
    const double mt = p2(t);
    if (mt != 0.) t = scale(t, 1. / sqrt(mt));
    int i0 = 1, i1 = 2, i2 = 3;
    const double ml[4] = {0., fabs(l.x), fabs(l.y), fabs(l.z)};
    if (ml[i2] > ml[i1]) { const int s = i1; i1 = i2; i2 = s; }
    if (ml[i1] > ml[i0]) { const int s = i0; i0 = i1; i1 = s; }
    if (ml[i2] > ml[i1]) { const int s = i1; i1 = i2; i2 = s; }
    const double tdp = comp(t, i1) * comp(l, i1) + comp(t, i2) * comp(l, i2);
    if (tdp != 0.) set_comp(t, i0, -tdp / comp(l, i0));
    if (p2(t) == 0.) set_comp(t, i1, 1.);
    return t;
}

// Poincare boost with m_l = l, m_rsq = rsq (Poincare.cc:36-50).
__device__ __forceinline__ V4 boost(V4 l, double rsq, V4 v) {
    const double lv = l.x * v.x + l.y * v.y + l.z * v.z;
    const double v0 = (l.e * v.e - lv) / rsq;
    const double c1 = (v.e + v0) / (rsq + l.e);
    return V4{v0, v.x - l.x * c1, v.y - l.y * c1, v.z - l.z * c1};
}
__device__ __forceinline__ V4 boost_back(V4 l, double rsq, V4 v) {
    const double lv = l.x * v.x + l.y * v.y + l.z * v.z;
    const double v0 = (l.e * v.e + lv) / rsq;
    const double c1 = (v.e + v0) / (rsq + l.e);
    return V4{v0, v.x + l.x * c1, v.y + l.y * c1, v.z + l.z * c1};
}

// SmallOMCT / SmallMLDP (FourVector.cc:57-69).
__device__ __forceinline__ double small_omct(V4 a, V4 v) {
    const double mag = sqrt(p2(a) * p2(v));
    const double pq = dot3(a, v);
    const double ct = std_min(std_max(pq / mag, -1.), 1.);
    if (ct < 0.) return 1. - ct;
    const double cx = a.y * v.z - a.z * v.y, cy = a.z * v.x - a.x * v.z, cz = a.x * v.y - a.y * v.x;
    const double st = sqrt(cx * cx + cy * cy + cz * cz) / mag;
    const double st2 = st / (2. * sqrt((ct + 1) / 2.));
    return 2. * st2 * st2;
}

// Isotropic two-body decay p -> p1 p2 (SChannelMomenta, ChannelElements.cc:87-111),
// ctmin = -1, ctmax = 1, reference axis (1,1,0,0).
__device__ __forceinline__ void schannel_momenta(V4 p, double s1, double s2, V4 &p1, V4 &p2o,
                                                 double ran1, double ran2) {
    const double s = mass2(p), rs = sqrt(fabs(s));
    const double e1 = (s + s1 - s2) / rs / 2., m1 = sqrt(e1 * e1 - s1);
    const double ct = -1. + 2. * ran1, st = sqrt(1. - ct * ct);
    const double ph = kTwoPi * ran2;
    const V4 xref{1., 1., 0., 0.};
    const V4 pl = p2(p) != 0. ? p : V4{1., 0., 0., 1.};
    const double rsq = sqrt(mass2(p));  // Poincare(p): m_rsq = p.Mass()
    const V4 n_perp = rotation_axis(pl, xref);
    V4 l_perp = lorentz_cross(pl, xref, n_perp);
    l_perp = scale(l_perp, 1.0 / sqrt(fabs(mass2(l_perp))));
    const double plp = sqrt(p2(pl));
    const double mc = m1 * ct;
    V4 q{e1, pl.x * mc / plp, pl.y * mc / plp, pl.z * mc / plp};
    const double cph = cos(ph), sph = sin(ph);
    q = q + scale(scale(l_perp, cph) + scale(n_perp, sph), m1 * st);
    q = boost_back(p, rsq, q);
    p1 = q;
    p2o = p - q;
}

// SChannelWeight (ChannelElements.cc:113-135): returns the weight, writes the
// two uniforms.
__device__ __forceinline__ double schannel_weight(V4 p1, V4 p2v, double &ran1, double &ran2) {
    const V4 p = p1 + p2v;
    const V4 pl = p2(p) != 0. ? p : V4{1., 0., 0., 1.};
    const V4 xref{1., 1., 0., 0.};
    const double rsq = sqrt(mass2(p));
    const V4 n_perp = rotation_axis(pl, xref);
    V4 l_perp = lorentz_cross(pl, xref, n_perp);
    l_perp = scale(l_perp, 1.0 / sqrt(fabs(mass2(l_perp))));
    const V4 p1h = boost(p, rsq, p1);
    const double ct = dot3(p1h, pl) / sqrt(p2(p1h) * p2(pl));
    double cp = -dot4(l_perp, p1), sp = -dot4(n_perp, p1);
    const double norm = sqrt(cp * cp + sp * sp);
    cp /= norm;
    sp /= norm;
    ran1 = (ct + 1.) / 2.;
    ran2 = atan2(sp, cp) / kTwoPi;
    if (ran2 < 0.) ran2 += 1.;
    double w = 1.;  // (ctmax - ctmin)/2
    const double s1 = std_max(mass2(p1), 0.), s2 = std_max(mass2(p2v), 0.);
    double s = mass2(p);
    if (s1 == 0. && s2 == 0.) s = p1.e * p2v.e * small_omct(p1, p2v);
    w *= sq_lambda(s, s1, s2) / (8. * kPi);
    return w;
}

// ------------------------------------------------- FSMapper forward
// FSMapper::GeneratePoint (Channel.cc:22-38): x[ndims] -> mom[slot] for all
// slots; mom[0..n_ext) are the external legs (incoming with negative energy).
__device__ __forceinline__ void fs_generate(const ChannelProgram *__restrict__ P, const double *x,
                                            V4 *mom, double *m2) {
    const int n_ext = P->n_ext;
    for (int s = 0; s < P->n_slots; ++s) m2[s] = P->slot_m2[s];
    int ir = 0;
    // GenDecays (Channel.cc:63-81)
    const int nd = P->n_decay;
    for (int k = 0; k < nd; ++k) {
        const int c1 = P->dec_c1[k], c2 = P->dec_c2[k];
        const double r = sqrt(m2[c1]) + sqrt(m2[c2]);
        const double smin1 = r * r;
        const double smin = std_max(std_max(smin1, P->dec_smin2[k]), P->dec_cut_smin[k]);
        const double smax = P->dec_smax[k];
        const double u = x[ir++];
        m2[P->dec_parent[k]] = P->dec_massless[k]
                                   ? massless_prop_momenta(0.99, smin, smax, u)
                                   : massive_prop_momenta(P->dec_mass[k], P->dec_width[k], smin, smax, u);
    }
    // GenTChan (Channel.cc:115-158)
    const double sqrts = P->sqrts, ptmax = P->ptmax;
    V4 psum{0., 0., 0., 0.};
    const int ni = P->n_info;
    for (int i = 0; i < ni - 1; ++i) {
        const double ptmin = P->info_ptmin[i];
        const double ran = x[ir++];
        const double pt = 2 * ptmin * ptmax * ran / (2 * ptmin + ptmax * (1 - ran));
        double etamax = sqrts / 2 / pt;
        etamax = log(etamax + sqrt(etamax * etamax - 1));
        etamax = std_min(etamax, P->info_etamax[i]);
        const double y = etamax * (2 * x[ir++] - 1);
        const double sinhy = sinh(y);
        const double coshy = sqrt(1 + sinhy * sinhy);
        const double ph = kTwoPi * x[ir++];
        const int sl = P->info_slot[i];
        const double mt = sqrt(pt * pt + m2[sl]);
        mom[sl] = V4{mt * coshy, pt * cos(ph), pt * sin(ph), mt * sinhy};
        psum = psum + mom[sl];
    }
    {
        const int sl = P->info_slot[ni - 1];
        const double mjets2 = mass2(psum);
        const double yjets = rapidity(psum);
        const double ptj2 = pt2(psum);
        const double qt = sqrt(m2[sl] + ptj2);
        const double mt = sqrt(mjets2 + ptj2);
        const double ymin = -log(sqrts / qt * (1 - mt / sqrts * exp(-yjets)));
        const double ymax = log(sqrts / qt * (1 - mt / sqrts * exp(yjets)));
        const double dely = ymax - ymin;
        const double yv = ymin + x[ir++] * dely;
        const double sinhy = sinh(yv);
        const double coshy = sqrt(1 + sinhy * sinhy);
        mom[sl] = V4{qt * coshy, -psum.x, -psum.y, qt * sinhy};
        const V4 tot = mom[sl] + psum;
        const double pp = tot.e + tot.z, pm = tot.e - tot.z;
        mom[0] = V4{-pp / 2, 0, 0, -pp / 2};
        mom[1] = V4{-pm / 2, 0, 0, pm / 2};
    }
    // GenSChan / DecayParts (Channel.cc:204-245)
    const int ns = P->n_sdec;
    for (int k = 0; k < ns; ++k) {
        const int a = P->sdec_a[k], b = P->sdec_b[k];
        const double r1 = x[ir++];
        const double r2 = x[ir++];
        schannel_momenta(mom[P->sdec_ab[k]], m2[a], m2[b], mom[a], mom[b], r1, r2);
    }
    (void)n_ext;
}

// ------------------------------------------------- FSMapper inverse
// FSMapper::GenerateWeight (Channel.cc:40-61).  mom[0..n_ext) holds the
// point; compound slots are rebuilt here.  Writes the uniforms into x in the
// reference's order; when the t-channel part fails (Channel.cc:197) it returns
// 0 without writing its last uniform, and the s-channel uniforms that follow
// shift down by one, exactly as in the reference.
__device__ __forceinline__ double fs_weight(const ChannelProgram *__restrict__ P, V4 *mom, double *x) {
    const int nd = P->n_decay;
    for (int k = 0; k < nd; ++k) mom[P->dec_parent[k]] = mom[P->dec_c1[k]] + mom[P->dec_c2[k]];
    int ir = 0;
    // WgtDecays (Channel.cc:83-113)
    double wdec = 1;
    for (int k = 0; k < nd; ++k) {
        const V4 a = mom[P->dec_c1[k]], b = mom[P->dec_c2[k]];
        const double r = sqrt(fabs(mass2(a))) + sqrt(fabs(mass2(b)));
        const double smin1 = r * r;
        const double smin = std_max(std_max(smin1, P->dec_smin2[k]), P->dec_cut_smin[k]);
        const double smax = P->dec_smax[k];
        const double s = mass2(mom[P->dec_parent[k]]);
        double u;
        if (P->dec_massless[k])
            wdec *= massless_prop_weight(0.99, smin, smax, s, u);
        else
            wdec *= massive_prop_weight(P->dec_mass[k], P->dec_width[k], smin, smax, s, u);
        x[ir++] = u;
        wdec /= kTwoPi;
    }
    // WgtTChan (Channel.cc:115-158, inverse at :160-202)
    const double sqrts = P->sqrts, ptmax = P->ptmax;
    double wt = kTwoPi;
    V4 psum{0., 0., 0., 0.};
    const int ni = P->n_info;
    for (int i = 0; i < ni - 1; ++i) {
        const double ptmin = P->info_ptmin[i];
        const V4 q = mom[P->info_slot[i]];
        wt *= P->inv16pi3;
        const double pt = sqrt(pt2(q));
        const double f2 = 2 * ptmin + pt;
        wt *= pt * ptmax / 2 / ptmin / (2 * ptmin + ptmax) * (f2 * f2);
        x[ir++] = pt * (ptmax + 2 * ptmin) / (ptmax * (pt + 2 * ptmin));
        double etamax = sqrts / 2 / pt;
        etamax = log(etamax + sqrt(etamax * etamax - 1));
        etamax = isnan(etamax) ? 99 : etamax;
        etamax = std_min(etamax, P->info_etamax[i]);
        wt *= 2 * etamax * 2 * kPi;
        const double y = rapidity(q);
        const double ph = phi_0_2pi(q);
        x[ir++] = (y / etamax + 1) / 2;
        x[ir++] = ph / 2 / kPi;
        psum = psum + q;
    }
    {
        const V4 q = mom[P->info_slot[ni - 1]];
        const double mjets2 = mass2(psum);
        const double yjets = rapidity(psum);
        const double ptj2 = pt2(psum);
        const double m2 = mass2(q);
        const double qt = sqrt(m2 + ptj2);
        const double mt = sqrt(mjets2 + ptj2);
        const double yv = rapidity(q);
        const double ymin = -log(sqrts / qt * (1 - mt / sqrts * exp(-yjets)));
        const double ymax = log(sqrts / qt * (1 - mt / sqrts * exp(yjets)));
        const double dely = ymax - ymin;
        if (isnan(ymax) || isnan(ymin)) {
            wt = 0;
        } else {
            wt *= dely / sqrts / sqrts;
            x[ir++] = (yv - ymin) / dely;
        }
    }
    // WgtSChan / WgtDecayParts (Channel.cc:222-256): s-channel uniforms are
    // still written after a t-channel failure (the reference evaluates all
    // three factors before multiplying them).
    double ws = 1;
    const int ns = P->n_sdec;
    for (int k = 0; k < ns; ++k) {
        double r1, r2;
        ws *= schannel_weight(mom[P->sdec_a[k]], mom[P->sdec_b[k]], r1, r2);
        x[ir++] = r1;
        x[ir++] = r2;
    }
    return wdec * wt * ws;
}

}  // namespace chili_dev

namespace chili_dev {

// The (smin, smax)-only terms of decay weight k of a PointProgram (computed
// on the device so that they round as the per-point code would):
// massless: pow(smin, 0.01), pow(smax, 0.01); massive: atan((smin-m2)/mw),
// atan((smax-m2)/mw) (the PeakedWeight and Breit-Wigner weights,
// ChannelElements.cc:27-50 and 64-85).
__device__ __forceinline__ void pp_prepare_entry(PointProgram *__restrict__ pp, int k) {
    const double smin = pp->dw_smin_c[k], smax = pp->dw_smax[k];
    if (pp->dw_massless[k]) {
        const double ce = 1. - 0.99;
        pp->dw_t1[k] = pow(smin, ce);
        pp->dw_t2[k] = pow(smax, ce);
    } else {
        const double m2 = pp->dw_mass[k] * pp->dw_mass[k], mw = pp->dw_mass[k] * pp->dw_width[k];
        pp->dw_t1[k] = atan((smin - m2) / mw);  // "ymax" of ChannelElements.cc:94
        pp->dw_t2[k] = atan((smax - m2) / mw);  // "ymin"
    }
}

// Integrand::GenerateWeight (Integrand.hh:112-123) over a PointProgram: the
// shared parts of all channels are evaluated once per point, then every
// channel's density is assembled as the reference multiplies it
// (Channel.cc:40-61: WgtDecays * WgtTChan * WgtSChan, each in its own order)
// and its uniforms are written into the buffer x that all channels share
// (not cleared between channels, as the reference's _rans).  ext holds the
// external momenta; xs receives channel ich's uniforms; dens[c*stride] the
// per-channel densities.  Returns 1 / sum_c alpha_c / dens_c / vw_c.
__device__ __forceinline__ double combined_weight_pp(const PointProgram *__restrict__ pp,
                                                     const double *__restrict__ grids,
                                                     const double *__restrict__ alpha, int dims, int bins, int ich,
                                                     const V4 *ext, double *x, double *xs, double *dens,
                                                     int dens_stride, double before) {
    V4 nm[PP_MAX_NODES];
    const int ne = pp->n_ext, nn = pp->n_nodes;
    for (int i = 0; i < ne; ++i) nm[i] = ext[i];
    for (int i = ne; i < nn; ++i) nm[i] = nm[pp->node_a[i]] + nm[pp->node_b[i]];
    const double sqrts = pp->sqrts, ptmax = pp->ptmax;

    // t-channel entries (WgtTChan loop body, Channel.cc:160-186)
    double tfac[PP_MAX_TENTS], tg[PP_MAX_TENTS], tx0[PP_MAX_TENTS], tx1[PP_MAX_TENTS], tx2[PP_MAX_TENTS];
    const int nt = pp->n_tents;
    for (int t = 0; t < nt; ++t) {
        const double ptmin = pp->tent_ptmin[t];
        const V4 q = nm[pp->tent_node[t]];
        const double pt = sqrt(pt2(q));
        const double f2 = 2 * ptmin + pt;
        tfac[t] = pt * ptmax / 2 / ptmin / (2 * ptmin + ptmax) * (f2 * f2);
        tx0[t] = pt * (ptmax + 2 * ptmin) / (ptmax * (pt + 2 * ptmin));
        double etamax = sqrts / 2 / pt;
        etamax = log(etamax + sqrt(etamax * etamax - 1));
        etamax = isnan(etamax) ? 99 : etamax;
        etamax = std_min(etamax, pp->tent_etacut[t]);
        tg[t] = 2 * etamax * 2 * kPi;
        tx1[t] = (rapidity(q) / etamax + 1) / 2;
        tx2[t] = phi_0_2pi(q) / 2 / kPi;
    }
    // whole chains, last entry included (Channel.cc:186-202)
    double cw[PP_MAX_CHAINS], cx[PP_MAX_CHAINS];
    unsigned long long cfail = 0;
    const int nc = pp->n_chains;
    for (int c = 0; c < nc; ++c) {
        double wt = kTwoPi;
        V4 psum{0., 0., 0., 0.};
        const int len = pp->chain_len[c];
        for (int i = 0; i < len; ++i) {
            const int t = pp->chain_tent[c][i];
            wt *= pp->inv16pi3;
            wt *= tfac[t];
            wt *= tg[t];
            psum = psum + nm[pp->tent_node[t]];
        }
        const V4 q = nm[pp->chain_last[c]];
        const double mjets2 = mass2(psum);
        const double yjets = rapidity(psum);
        const double ptj2 = pt2(psum);
        const double qt = sqrt(mass2(q) + ptj2);
        const double mt = sqrt(mjets2 + ptj2);
        const double yv = rapidity(q);
        const double ymin = -log(sqrts / qt * (1 - mt / sqrts * exp(-yjets)));
        const double ymax = log(sqrts / qt * (1 - mt / sqrts * exp(yjets)));
        const double dely = ymax - ymin;
        if (isnan(ymax) || isnan(ymin)) {
            cfail |= 1ull << c;
            cw[c] = 0;
            cx[c] = 0;
        } else {
            cw[c] = wt * (dely / sqrts / sqrts);
            cx[c] = (yv - ymin) / dely;
        }
    }
    // decay propagator weights (WgtDecays, Channel.cc:83-113)
    double dw[PP_MAX_DWS], dx[PP_MAX_DWS];
    const int nd = pp->n_dws;
    for (int k = 0; k < nd; ++k) {
        const double r = sqrt(fabs(mass2(nm[pp->dw_c1[k]]))) + sqrt(fabs(mass2(nm[pp->dw_c2[k]])));
        const double smin = std_max(std_max(r * r, pp->dw_smin2[k]), pp->dw_cut[k]);
        const double s = mass2(nm[pp->dw_node[k]]);
        double u;
        dw[k] = pp->dw_massless[k] ? massless_prop_weight(0.99, smin, pp->dw_smax[k], s, u)
                                   : massive_prop_weight(pp->dw_mass[k], pp->dw_width[k], smin, pp->dw_smax[k], s, u);
        dx[k] = u;
    }
    // two-body decays (WgtDecayParts, Channel.cc:222-237)
    double sw[PP_MAX_SWS], sr1[PP_MAX_SWS], sr2[PP_MAX_SWS];
    const int ns = pp->n_sws;
    for (int k = 0; k < ns; ++k) sw[k] = schannel_weight(nm[pp->sw_a[k]], nm[pp->sw_b[k]], sr1[k], sr2[k]);

    for (int d = 0; d < dims; ++d) x[d] = 0.0;
    double acc = 0;
    const size_t gsz = static_cast<size_t>(dims) * (bins + 1);
    const int nch = pp->nch;
    for (int c = 0; c < nch; ++c) {
        const PPChannel &C = pp->ch[c];
        int ir = 0;
        double wdec = 1;
        for (int k = 0; k < C.n_dec; ++k) {
            wdec *= dw[C.dw[k]];
            x[ir++] = dx[C.dw[k]];
            wdec /= kTwoPi;
        }
        const int ch = C.chain;
        const int len = pp->chain_len[ch];
        for (int i = 0; i < len; ++i) {
            const int t = pp->chain_tent[ch][i];
            x[ir++] = tx0[t];
            x[ir++] = tx1[t];
            x[ir++] = tx2[t];
        }
        if (!((cfail >> ch) & 1ull)) x[ir++] = cx[ch];
        double ws = 1;
        for (int k = 0; k < C.n_sd; ++k) {
            ws *= sw[C.sw[k]];
            x[ir++] = sr1[C.sw[k]];
            x[ir++] = sr2[C.sw[k]];
        }
        const double dc = wdec * cw[ch] * ws;
        if (c == ich)
            for (int d = 0; d < dims; ++d) xs[d] = x[d];
        const double vw = grid_weight(grids + c * gsz, dims, bins, x, before);
        acc += __ldg(alpha + c) / dc / vw;
        if (dens) dens[static_cast<size_t>(c) * dens_stride] = dc;
    }
    return 1.0 / acc;
}

}  // namespace chili_dev
