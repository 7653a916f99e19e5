"""The reference's MPI mode on several GPUs: every rank integrates its own
points (its own counter range), then the ranks sum their training data and
StatsData with one all-reduce and every rank adapts identically.

Reference: MultiChannel::operator() splits ncalls over the ranks and, before
Train, all-reduces the per-channel histograms, the alpha-training sums and
the StatsData (include/Channel/MultiChannel.hh:184-212, Vegas.cc:24-47 for
plain VEGAS). Here one rank = one process = one GPU; the exchange is one
`torch.distributed.all_reduce` (NCCL over NVLink on GPUs, gloo on CPU) of a
packed FP64 buffer [histograms | alpha training | n, sum, sum2, n_finite]
plus one MAX all-reduce of the StatsData maximum and minimum. Integrators plug in through a
three-method interface:

    run(params)       one iteration that collects its training data but does
                      not train (the library's "defer_train" option) ->
                      (stats tuple, info)
    training()        (hist [nch, dims, bins], alpha_train [nch]) arrays or tensors
    train(params, hist, alpha_train)   adapt from the summed training data
"""
import numpy as np


def pack(hist, atrain, stats):
    """[hist | atrain | n, sum, sum2, n_finite] in one FP64 vector."""
    st = np.asarray(stats, dtype=np.float64)
    return np.concatenate([np.asarray(hist, dtype=np.float64).ravel(), np.asarray(atrain, dtype=np.float64).ravel(),
                           st[[0, 3, 4, 5]]])


def unpack(buf, hist_shape, nch):
    nh = int(np.prod(hist_shape))
    hist = buf[:nh].reshape(hist_shape)
    atrain = buf[nh:nh + nch]
    n, s, s2, nf = buf[nh + nch:nh + nch + 4]
    return hist, atrain, (n, 0.0, 0.0, s, s2, nf)


def synced_iteration(integrator, params, group=None, device=None):
    """One iteration of the MPI mode on this rank: local points, one
    all-reduce of the training data and StatsData, identical training on
    every rank. Returns the merged StatsData tuple (n, min, max, sum, sum2,
    n_finite) and this rank's iteration record.

    A rank that packs its training data on the device (GpuRank with a CUDA
    device) exchanges it in place: the library writes the packed buffer on
    the device, the all-reduce runs on it (NCCL over NVLink), and the
    library trains from device pointers into the summed buffer; only the six
    merged StatsData values come back to the host."""
    import torch
    import torch.distributed as dist
    if device is not None and torch.device(device).type == "cuda" and hasattr(integrator, "pack_training"):
        st, info = integrator.run(params)
        buf = integrator.pack_training(device)
        nh = buf.shape[0] - 6 - integrator.nch
        dist.all_reduce(buf[:-2], group=group)
        dist.all_reduce(buf[-2:], op=dist.ReduceOp.MAX, group=group)
        integrator.train(params, buf[:nh], buf[nh:nh + integrator.nch])
        s = buf[-6:].cpu().numpy()
        return (s[0], -float(s[5]), float(s[4]), s[1], s[2], s[3]), info
    st, info = integrator.run(params)
    hist, atrain = integrator.training()
    hist = np.asarray(hist, dtype=np.float64)
    atrain = np.asarray(atrain, dtype=np.float64)
    buf = torch.from_numpy(pack(hist, atrain, st))
    ext = torch.tensor([float(st[2]), -float(st[1])], dtype=torch.float64)  # max, -min
    if device is not None:
        buf, ext = buf.to(device), ext.to(device)
    dist.all_reduce(buf, group=group)
    dist.all_reduce(ext, op=dist.ReduceOp.MAX, group=group)
    h, a, merged = unpack(buf.cpu().numpy(), hist.shape, atrain.size)
    integrator.train(params, h, a)
    e = ext.cpu().numpy()
    merged = (merged[0], -float(e[1]), float(e[0]), merged[3], merged[4], merged[5])
    return merged, info


class GpuRank:
    """A chili_b200 context as one rank (its own seed or counter range).
    shared_stream: the context runs on torch's current stream (set with
    Context.set_stream), so the collectives and the library's kernels are
    ordered by the stream alone; otherwise the two streams are synchronised
    around the collective."""

    def __init__(self, ctx, seed, counter, shared_stream=False):
        self.ctx, self.seed, self.counter = ctx, seed, counter
        self.shared_stream = shared_stream
        ctx.set_option("defer_train", 1)

    def run(self, params):
        st, info = self.ctx.multichannel_iterate(params, seed=self.seed, counter=self.counter)
        self.counter += info.points_tried
        return st.as_tuple(), info

    @property
    def nch(self):
        return self.ctx.nch

    def training(self):
        return self.ctx.get_training()

    def pack_training(self, device):
        """The packed training buffer in device memory (chili_gpu_pack_training)."""
        import torch
        buf = torch.empty(self.ctx.packed_training_len(), dtype=torch.float64, device=device)
        if not self.shared_stream:
            torch.cuda.current_stream(device).synchronize()  # buf's allocation, on torch's stream
        self.ctx.pack_training(buf)
        if not self.shared_stream:
            self.ctx.synchronize()
        return buf

    def train(self, params, hist, atrain):
        if not self.shared_stream and hasattr(hist, "device") and hist.device.type == "cuda":
            import torch
            torch.cuda.current_stream(hist.device).synchronize()  # the collective's result
        self.ctx.multichannel_train(params, hist, atrain)
