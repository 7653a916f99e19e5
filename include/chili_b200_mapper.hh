// chili_b200_mapper.hh -- the GPU phase-space mapping as the reference's own
// plugin type: chili::gpu::GpuFSMapper is a chili::Mapper<chili::FourVector>
// (Chili include/Channel/Mapper.hh:37-39), so a reference Channel<FourVector>
// (include/Channel/Integrand.hh:9-16) holds it in its unique_ptr<Mapper>
// slot in place of chili::FSMapper (include/Channel/Channel.hh:15-33), and the
// reference's Integrand / MultiChannel drive it unchanged.
//
// Compiled only where Chili's own headers are on the include path (the
// class derives from Chili's Mapper and takes its ChannelDescription and
// Cuts); without them this header declares nothing.  Link against
// libchili_b200 and the Chili library as before.
//
// Each call maps one point on the GPU (one upload, one kernel, one read-back):
// the per-point plugin surface of the reference.  Code that maps many points
// at once uses chili_gpu_fsmapper_generate / chili_gpu_fsmapper_weight on
// whole batches, or the multichannel iteration, instead.
#pragma once

#if __has_include("Channel/Mapper.hh") && __has_include("Channel/Channel.hh")

#include <map>
#include <memory>
#include <ostream>
#include <string>
#include <utility>
#include <vector>

#include "Channel/Channel.hh"
#include "Channel/Mapper.hh"
#include "Tools/Cuts.hh"
#include "Tools/FourVector.hh"
#include "chili_b200.hh"

namespace chili {
namespace gpu {

class GpuFSMapper : public chili::Mapper<chili::FourVector> {
  public:
    // FSMapper(sqrts, ntot, ChannelDescription, Cuts) (Channel.hh:18-30):
    // the channel is flattened into a device program on `device`.  Throws
    // chili::gpu::Error when the description is inconsistent (a missing
    // cut entry, which the reference's constructor reports by
    // std::out_of_range from Cuts::ptmin.at).
    GpuFSMapper(double sqrts, size_t ntot, chili::ChannelDescription channel, chili::Cuts cuts, int device = 0)
        : sqrts_(sqrts), ntot_(ntot), channel_(std::move(channel)), cuts_(std::move(cuts)), ctx_(device) {
        chili::gpu::ChannelDescription d;
        for (const auto &p : channel_.info) d.info.push_back(conv(p));
        for (const auto &kv : channel_.decays)  // DecayMap order (ParticleInfo operator<)
            d.decays.push_back({conv(kv.first), {conv(kv.second.first), conv(kv.second.second)}});
        chili::gpu::Cuts c;
        c.sexternal = cuts_.sexternal;
        c.deltaR = cuts_.deltaR;
        for (const auto &kv : cuts_.smin) c.smin[kv.first] = kv.second;
        for (const auto &kv : cuts_.ptmin) c.ptmin[kv.first] = kv.second;
        for (const auto &kv : cuts_.etamax) c.etamax[kv.first] = kv.second;
        set_ = std::make_unique<ChannelSet>(std::vector<chili::gpu::ChannelDescription>{d}, c, sqrts_,
                                            static_cast<int>(ntot_));
        check(chili_gpu_set_channels(ctx_.get(), set_->descs(), 1, set_->cuts(), sqrts_, static_cast<int>(ntot_)),
              ctx_.get());
        ndims_ = static_cast<size_t>(chili_gpu_ndims(ctx_.get()));
        for (const auto &p : channel_.info) ptmin_.push_back(cuts_.ptmin.at(p.idx) != 0 ? cuts_.ptmin.at(p.idx) : 1);
    }

    // FSMapper::GeneratePoint (Channel.cc:22-38): rans[NDims()] -> ntot
    // momenta, incoming legs with negative energy.
    void GeneratePoint(std::vector<chili::FourVector> &mom, const std::vector<double> &rans) override {
        if (rans.size() < ndims_) throw Error(CHILI_ERR_INVALID_ARG, "GpuFSMapper: fewer uniforms than NDims()");
        mom_buf_.resize(4 * ntot_);
        check(chili_gpu_fsmapper_generate(ctx_.get(), 0, rans.data(), mom_buf_.data(), 1), ctx_.get());
        mom.resize(ntot_);
        for (size_t i = 0; i < ntot_; ++i)
            mom[i] = chili::FourVector(mom_buf_[4 * i], mom_buf_[4 * i + 1], mom_buf_[4 * i + 2], mom_buf_[4 * i + 3]);
    }

    // FSMapper::GenerateWeight (Channel.cc:40-61): the channel density of
    // the momenta; the uniforms of the inverse map land in rans, which is an
    // in/out buffer as in the reference (entries the map does not consume
    // keep their contents; Integrand::GenerateWeight shares one buffer
    // between the channels, Integrand.hh:112-123).
    double GenerateWeight(const std::vector<chili::FourVector> &mom, std::vector<double> &rans) override {
        if (mom.size() < ntot_) throw Error(CHILI_ERR_INVALID_ARG, "GpuFSMapper: fewer momenta than legs");
        mom_buf_.resize(4 * ntot_);
        for (size_t i = 0; i < ntot_; ++i)
            for (size_t k = 0; k < 4; ++k) mom_buf_[4 * i + k] = mom[i][k];
        if (rans.size() < ndims_) rans.resize(ndims_, 0.0);
        double w = 0;
        check(chili_gpu_fsmapper_weight_inout(ctx_.get(), 0, mom_buf_.data(), rans.data(), &w, 1), ctx_.get());
        return w;
    }

    // 3 n_out - 4 + 2 (Channel.hh:33)
    size_t NDims() const override { return ndims_; }

    static std::string Name() { return "FSMapper"; }

  private:
    static chili::gpu::ParticleInfo conv(const chili::ParticleInfo &p) {
        return chili::gpu::ParticleInfo{p.idx, p.pid, p.mass, p.width};
    }
    // A checkpoint (MultiChannel::SaveAs, MultiChannel.cc:79-107) stores this
    // mapper as an FSMapper in the reference's own layout (Channel.cc:7-20),
    // so the file loads back as a stock FSMapper.
    std::string GetName() const override { return Name(); }
    bool _Serialize(std::ostream &out) const override {
        channel_.Serialize(out);
        const double ptmax = sqrts_ / 2.0;
        const size_t nout = ntot_ - 2, size = ptmin_.size();
        out.write(reinterpret_cast<const char *>(&sqrts_), sizeof(sqrts_));
        out.write(reinterpret_cast<const char *>(&ptmax), sizeof(ptmax));
        out.write(reinterpret_cast<const char *>(&ntot_), sizeof(ntot_));
        out.write(reinterpret_cast<const char *>(&nout), sizeof(nout));
        out.write(reinterpret_cast<const char *>(&size), sizeof(size));
        for (const double pt : ptmin_) out.write(reinterpret_cast<const char *>(&pt), sizeof(pt));
        return true;
    }

    double sqrts_;
    size_t ntot_, ndims_{};
    chili::ChannelDescription channel_;
    chili::Cuts cuts_;
    std::vector<double> ptmin_;
    Context ctx_;
    std::unique_ptr<ChannelSet> set_;
    std::vector<double> mom_buf_;
};

}  // namespace gpu
}  // namespace chili

#endif
