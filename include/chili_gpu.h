/*
 * chili_gpu.h -- C ABI of the B200 implementation of Chili's integration hot
 * path: VEGAS point generation and grid adaptation, and the multichannel
 * t/s-channel phase-space mappings (FSMapper), with the combined channel
 * weight and channel-weight adaptation.
 *
 * Every entry point is extern "C", takes plain pointers and sizes, and returns
 * a status code (CHILI_OK == 0).  No exception crosses the boundary; the text
 * of the last error is available from chili_gpu_last_error().
 *
 * Pointer arguments marked "host or device" may point to host memory (pageable
 * or pinned) or to device memory of the context's GPU; the library detects
 * which through CUDA unified addressing and stages host buffers through its own
 * device buffers.  All work of a context is issued on one CUDA stream; a
 * context must not be used from two host threads at the same time.
 *
 * Reference interfaces replaced (paths inside the Chili project):
 *   AdaptiveMap   include/Integrator/AdaptiveMap.hh:26-73, src/Integrator/AdaptiveMap.cc:34-160
 *   Vegas         include/Integrator/Vegas.hh:30-95, src/Integrator/Vegas.cc:18-82
 *   StatsData     include/Integrator/Statistics.hh:62-142
 *   FSMapper      include/Channel/Channel.hh:15-77, src/Channel/Channel.cc:22-256
 *   Integrand     include/Channel/Integrand.hh:107-123
 *   MultiChannel  include/Channel/MultiChannel.hh:29-251, src/Channel/MultiChannel.cc:109-154
 *   Interface::Evaluate (nanobind) include/Interfaces/nanobind.hh:23-50
 *   CallChili (TensorFlow op)      src/Interfaces/Tensorflow.cc:22-135
 */
#ifndef CHILI_GPU_H
#define CHILI_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
enum chili_status {
    CHILI_OK = 0,
    CHILI_ERR_INVALID_ARG = 1, /* bad pointer, size or description          */
    CHILI_ERR_CUDA = 2,        /* a CUDA runtime call failed                */
    CHILI_ERR_TIMEOUT = 3,     /* a bounded device wait gave up             */
    CHILI_ERR_NAN_GRID = 4,    /* adaptation produced a non-finite edge     */
    CHILI_ERR_STATE = 5,       /* call made before the state it needs       */
    CHILI_ERR_LIMIT = 6        /* size beyond a compiled limit (see below)  */
};

/* ---------------------------------------------------------------- limits */
#define CHILI_MAX_EXT 10      /* external particles, incoming included     */
#define CHILI_MAX_DIMS 32     /* integration dimensions per channel        */
#define CHILI_MAX_CHANNELS 200
#define CHILI_MAX_BINS 4096   /* VEGAS bins per dimension                  */
#define CHILI_MAX_INTEGRAND_PARAMS 128

/* ------------------------------------------------------- phase-space data */
/* ParticleInfo (include/Channel/ChannelNode.hh:26-32): idx is the bitmask of
 * external legs (leg i <-> 1<<i; legs 0 and 1 are incoming). */
typedef struct {
    uint32_t idx;
    int32_t pid;
    double mass;
    double width;
} chili_particle_info;

/* One DecayMap entry (ChannelNode.hh:35): parent -> (child1, child2). */
typedef struct {
    chili_particle_info parent, child1, child2;
} chili_decay;

/* ChannelDescription (ChannelNode.hh:46-51).  info is the t-channel list in
 * the caller's order (the last entry balances momentum); decays may come in
 * any order: they are processed in the reference's std::map order, i.e.
 * ascending (idx, mass, width) of the parent. */
typedef struct {
    int32_t n_info;
    const chili_particle_info *info;
    int32_t n_decays;
    const chili_decay *decays;
} chili_channel_desc;

typedef struct {
    uint32_t idx;
    double value;
} chili_idx_value;

typedef struct {
    int32_t pid1, pid2;
    double value;
} chili_pid_pair_value;

/* Cuts (include/Tools/Cuts.hh:13-19) as flat key/value tables.  sexternal
 * holds the squared masses of the outgoing legs.  Keys absent from smin read
 * as 0 and from deltaR as 0 (Channel.cc:148-151); ptmin and etamax must hold
 * every idx that the channel descriptions reference (Channel.hh:22,
 * Channel.cc:150,209). */
typedef struct {
    int32_t n_sexternal;
    const double *sexternal;
    int32_t n_deltaR;
    const chili_pid_pair_value *deltaR;
    int32_t n_smin;
    const chili_idx_value *smin;
    int32_t n_ptmin;
    const chili_idx_value *ptmin;
    int32_t n_etamax;
    const chili_idx_value *etamax;
} chili_cuts;

/* ------------------------------------------------------------ statistics */
/* StatsData (Statistics.hh:62-142), same field order as its binary form. */
typedef struct {
    double n, min, max, sum, sum2, n_finite;
} chili_stats;

/* MultiChannelParams (MultiChannel.hh:29-49) and its defaults. */
typedef struct {
    uint64_t ncalls;        /* 10000 */
    uint64_t niterations;   /* 10    */
    double rtol;            /* 1e-5  */
    uint64_t nrefine;       /* 1     */
    double beta;            /* 0.25  */
    double min_alpha;       /* 1e-5  */
    double refine_size;     /* 1.5   */
    uint64_t max_bins;      /* 200   */
    uint64_t iteration;     /* 0     */
    int32_t should_optimize;/* 1     */
    double grid_alpha;      /* VegasParams::alpha of every channel grid, 1.0 */
} chili_multichannel_params;

/* What one multichannel iteration did, besides its StatsData. */
typedef struct {
    uint64_t points_tried;    /* counters consumed (incl. rejected points)  */
    uint64_t points_accepted; /* == ncalls on success                       */
    uint64_t rejected_pre;    /* PreProcess rejections                      */
    uint64_t rejected_nan;    /* NaN-value retries (MultiChannel.hh:230-236)*/
    double weight_max;        /* max combined weight f*w over the iteration */
    double nonfinite_alpha_terms; /* non-finite alpha-training contributions */
    uint64_t points_weighted; /* points whose combined weight was computed
                                 (PreProcess-accepted points of the chunks,
                                 including those beyond the cut)           */
    uint64_t points_drawn;    /* counters the chunks' forward launches
                                 covered (each chunk is drawn whole,
                                 including points beyond the cut)          */
    uint64_t chunks;          /* chunks of points the iteration drew       */
} chili_mc_iter_info;

/* ------------------------------------------------------------ integrands */
enum chili_integrand_kind {
    /* f = 1 (the unit integrand of src/example.cc:120-122). */
    CHILI_FUNC_UNIT = 0,
    /* f(x) = N [exp(-|x-a|^2/s^2) + exp(-|x-b|^2/s^2)] over [0,1]^D.
     * params = {s, N, a[0..D-1], b[0..D-1]}, D = grid dimensions. */
    CHILI_FUNC_CAMEL = 1,
    /* Sum over outgoing pairs (i<j) of 1/((s_ij-M^2)^2+M^2 G^2) times the
     * product over outgoing j of 1/(|t_0j|+m^2), t_0j = (p_0+p_j)^2 in the
     * all-outgoing convention.  params = {M, G, m}. */
    CHILI_FUNC_PROPAGATOR = 2,
    /* As CHILI_FUNC_PROPAGATOR but the product of the two largest pair
     * factors instead of their sum.  params = {M, G, m}. */
    CHILI_FUNC_PROPAGATOR_TOP2 = 3
};

/* PreProcess cut applied to every generated point (MultiChannel.hh:219-223). */
enum chili_preprocess_kind {
    CHILI_PRE_ACCEPT_ALL = 0,
    /* reject when the first momentum's energy is NaN (src/example.cc:26-29) */
    CHILI_PRE_FINITE = 1,
    /* the physical region and the usual cuts (set with
     * chili_gpu_set_preprocess_cuts): finite momenta, incoming energies
     * |E_0|, |E_1| <= sqrts/2 (momentum fractions <= 1), every outgoing leg
     * pT >= ptmin and |eta| <= etamax, every outgoing pair
     * Delta R = sqrt(Delta eta^2 + Delta phi^2) >= delta_r.  The reference's
     * FSMapper generates points outside this region (fractions above 1,
     * s-channel decay products below the pT cut) that its weights do not
     * describe consistently across channels; inside it every channel's
     * single-channel estimate agrees. */
    CHILI_PRE_CUTS = 2
};

/* ------------------------------------------------------------ context */
typedef struct chili_ctx chili_ctx;

/* Create a context on CUDA device `device`. */
int chili_gpu_create(int device, chili_ctx **out);
int chili_gpu_destroy(chili_ctx *ctx);
/* Last error text of ctx (or of the library when ctx is NULL). */
const char *chili_gpu_last_error(const chili_ctx *ctx);
/* Use the given cudaStream_t for all later work (NULL: the context's own). */
int chili_gpu_set_stream(chili_ctx *ctx, void *stream);
int chili_gpu_synchronize(chili_ctx *ctx);
/* Number of kernels this context has launched so far. */
uint64_t chili_gpu_launch_count(const chili_ctx *ctx);
/* Tuning switches (no counterpart in the reference).  "point_program": 1
 * (default) evaluates the parts that channels share once per point, 0 runs
 * every channel's mapping on its own; both give the same numbers.
 * "pipeline": 1 (default) runs the all-channel weight pass as a sequence of
 * small kernels over tiles of points, 0 as one kernel per point.
 * "pipeline_tile": points per tile of that pass (default 4194304).
 * "kernel_timing": 1 brackets the iteration's kernels with CUDA events on the
 * context's stream (totals read by chili_gpu_kernel_time; setting the option
 * resets them), 0 (default) records nothing.
 * "defer_train": 1 makes an optimizing iteration collect its training data
 * without applying Train, for a caller that sums the data over ranks first
 * and then calls chili_gpu_multichannel_train (the reference's MPI mode);
 * 0 (default) trains at the end of the iteration.
 * "max_rounds": chunks of points a multichannel iteration may draw before it
 * gives up with CHILI_ERR_TIMEOUT (default 100000; the reference's loop has
 * no such bound and never ends when every point is rejected or NaN).
 * "batch_phased": 1 (default) weights the batched multichannel tasks whose
 * channel set has a shared-entry program with the phased weight pass (task
 * chains as parallel graph branches); 0 evaluates every point in one thread
 * of the persistent batch kernel.  Read by chili_gpu_batch_set.
 * "batch_retry": 1 keeps the reference's retry loop for batched multichannel
 * tasks (MultiChannel.hh:214-248: points are drawn until ncalls of them pass
 * PreProcess with a finite value, the others count as zero-valued calls), in
 * rounds; an iteration that still lacks points after max_rounds further
 * rounds fails with CHILI_ERR_TIMEOUT (the reference's loop never ends on a
 * task whose values are all NaN).  It needs the grouped phased pass
 * (batch_grouped and batch_phased on; chili_gpu_batch_set fails otherwise).
 * 0 (default): a fixed budget of ncalls drawn points per task and iteration,
 * rejected points and NaN values counting as zero-valued calls.  Read by
 * chili_gpu_batch_set.
 * "channel_tables": 1 (default) stages each channel's edge, hint and width
 * tables in shared memory for the bin searches of the phased weight pass
 * (tables up to 112 KB), 0 reads them from global memory; the same numbers.
 * "flow_streamed": 1 runs a learned proposal of 2 x 128 hidden units on the
 * streamed-weight coupling kernels that wider or deeper conditioners always
 * use (the same function; a cross-check of the two kernel families), 0
 * (default) on the kernels that keep the weights in shared memory.  Read by
 * chili_gpu_flow_init. */
int chili_gpu_set_option(chili_ctx *ctx, const char *name, int64_t value);
/* Total device time (ms) and launch count of one kernel class under the
 * "kernel_timing" option: k_mc_forward, k_pp_nodes, k_pp_items, k_pp_chains,
 * k_pp_channel, k_pp_combine, k_mc_weight, k_mc_accum, k_vegas_iter.  No
 * counterpart in the reference. */
int chili_gpu_kernel_time(chili_ctx *ctx, const char *kernel, double *ms, uint64_t *launches);

/* ------------------------------------------------- grids (AdaptiveMap) */
/* nch grids of dims x (bins+1) edges, each in the reference AdaptiveMap
 * layout edges[dim*(bins+1)+k] (AdaptiveMap.hh:29-40,47-48).  Host or device. */
int chili_gpu_set_grids(chili_ctx *ctx, const double *edges, int nch, int dims,
                        int bins);
int chili_gpu_get_grids(chili_ctx *ctx, double *edges, int nch, int dims,
                        int bins);
/* AdaptiveMap::operator() (AdaptiveMap.cc:40-56) on n points of grid ch:
 * u[n*dims] -> x[n*dims], jac[n].  Host or device. */
int chili_gpu_grid_map(chili_ctx *ctx, int ch, const double *u, double *x,
                       double *jac, int64_t n);
/* AdaptiveMap::FindBin (:34-38) and ::GenerateWeight (:58-65): x[n*dims] ->
 * w[n] and (optional) bin[n*dims]; a FindBin of SIZE_MAX reads as -1. */
int chili_gpu_grid_weight(chili_ctx *ctx, int ch, const double *x, double *w,
                          int32_t *bin, int64_t n);
/* AdaptiveMap::Adapt (:67-125) of grid ch with damping alpha from
 * train[dims*bins].  Host or device. */
int chili_gpu_grid_adapt(chili_ctx *ctx, int ch, double alpha,
                         const double *train);
/* AdaptiveMap::Split (:127-160) of every grid into nsplit (2, 3 or 4). */
int chili_gpu_grid_split(chili_ctx *ctx, int nsplit);

/* ------------------------------------------------------------ integrand */
int chili_gpu_set_integrand(chili_ctx *ctx, int kind, const double *params,
                            int nparams);
int chili_gpu_set_preprocess(chili_ctx *ctx, int kind);
/* PreProcess = CHILI_PRE_CUTS with these cut values (channels must be set:
 * the cuts apply to their external legs). */
int chili_gpu_set_preprocess_cuts(chili_ctx *ctx, double sqrts, double ptmin, double etamax, double delta_r);

/* ------------------------------------------------------ plain VEGAS */
/* One Vegas::operator() (Vegas.cc:18-52) on grid 0: ncalls points, uniforms
 * from the counter-based generator (seed, counter_base + i) or, when u is not
 * NULL, from u[ncalls*dims]; f*J accumulated into stats_out, f^2 J^2 into the
 * per-bin training histogram (copied to train_out[dims*bins] when not NULL),
 * and, when adapt != 0, AdaptiveMap::Adapt(alpha) applied to grid 0. */
int chili_gpu_vegas_iterate(chili_ctx *ctx, uint64_t ncalls, uint64_t seed,
                            uint64_t counter_base, const double *u,
                            double alpha, int adapt, chili_stats *stats_out,
                            double *train_out);

/* Materialised VEGAS points (the events of a Vegas integration of the camel,
 * Vegas.cc:29-36 without the accumulation): point i takes the uniforms of
 * counter counter_base + i (the stream chili_gpu_vegas_iterate draws), maps
 * them through grid 0 (AdaptiveMap::operator(), AdaptiveMap.cc:40-56) and
 * writes x_out[i*dims + d] and its weight w_out[i] = f(x) J (NaN where a
 * uniform lies outside [0, 1)).  Host or device buffers.  The grid must fit
 * the kernel's shared-memory staging (8 dims (bins+1) + 8 * 256 (dims+1)
 * bytes <= 200 KB, else CHILI_ERR_LIMIT). */
int chili_gpu_vegas_generate(chili_ctx *ctx, uint64_t n, uint64_t seed, uint64_t counter_base, double *x_out,
                             double *w_out);

/* Plain VEGAS without any device allocation.  This entry point has no
 * counterpart in the reference.  It is for callers that cannot call
 * cudaMalloc: code running inside another framework whose device memory that
 * framework's allocator owns, or processes whose device-memory budget is fixed
 * before they start.  It creates no context: the caller passes the grid
 * (edges[dims*(bins+1)], the AdaptiveMap layout), the camel parameters (host
 * array {s, N, a[dims], b[dims]}) and the outputs, all on the current device.
 * The work of one Vegas::operator() without the adaptation runs on `stream`
 * (NULL: the legacy default stream): stats_out[6] receives the iteration's
 * StatsData and train_out[dims*bins] its f^2 J^2 histogram, the same numbers
 * as chili_gpu_vegas_iterate (histogram sums up to the order of addition).
 * Its scratch -- the integrand descriptor and the per-block partial sums, at
 * most 1184 blocks -- lives in one fixed array of about 57 KB that the library
 * declares in device memory, so every GPU that loads the library holds it until
 * the process exits.  The first call on a device looks up that array's address
 * (cudaGetSymbolAddress); make that first call before any stream capture.  All
 * calls share the array: calls whose work overlaps on the GPU race and must be
 * ordered by the caller (one stream, or events).  Limits: dims <= CHILI_MAX_DIMS,
 * 2 <= bins <= CHILI_MAX_BINS, 2 + 2*dims <= nparams <= CHILI_MAX_INTEGRAND_PARAMS,
 * 2 <= ncalls <= 2^40; larger sizes return CHILI_ERR_LIMIT. */
int chili_gpu_vegas_iterate_noalloc(void *stream, const double *edges, int dims, int bins,
                                    const double *camel_params, int nparams, uint64_t ncalls, uint64_t seed,
                                    uint64_t counter_base, double *stats_out, double *train_out);

/* ------------------------------------------------ channels (FSMapper) */
/* Build the device programs of nch FSMapper channels (Channel.hh:18-30) over
 * n_ext external legs at collider energy sqrts. */
int chili_gpu_set_channels(chili_ctx *ctx, const chili_channel_desc *descs,
                           int nch, const chili_cuts *cuts, double sqrts,
                           int n_ext);
/* Host-only check of channel descriptions (no device needed): 0 when the
 * channels are consistent (each consumes exactly 3*(n_ext-2)-2 uniforms,
 * every decaying current has its DecayMap entry, the cuts hold every key the
 * FSMapper reads with .at(), Channel.hh:22 and Channel.cc:150,209), else
 * CHILI_ERR_INVALID_ARG with the reason in err[err_len]. */
int chili_gpu_check_channels(const chili_channel_desc *descs, int nch, const chili_cuts *cuts, double sqrts,
                             int n_ext, char *err, size_t err_len);
/* ------------------------------------------------------ channel construction
 * ConstructChannels (src/Channel/ChannelNode.cc:74-291) on the host: the
 * FSMapper channel descriptions of a process from a model, to be passed to
 * chili_gpu_set_channels.  The Model (include/Model/Model.hh:10-29):
 * Combinable(f1, f2) is a callback that writes the flavours two currents
 * combine into (at most max_out) to out and returns their number (< 0:
 * error); masses and widths are keyed by |pid| and must hold every flavour
 * the enumeration meets (the reference's Model::Mass/Width use .at). */
typedef int (*chili_combinable_fn)(int32_t f1, int32_t f2, int32_t *out, int32_t max_out, void *user);
typedef struct {
    chili_combinable_fn combinable;
    void *user;
    int32_t n_masses;
    const chili_idx_value *masses;
    int32_t n_widths;
    const chili_idx_value *widths;
} chili_model;

typedef struct chili_channel_list chili_channel_list;

/* flavs[n_flavs]: the two incoming then the outgoing flavours (all-outgoing
 * convention, as the reference's flavs).  cuts == NULL: the first overload
 * (ChannelNode.cc:74-96: Delta R 0.4 between all flavours, 0 with a top;
 * pT > 30, |eta| < 99, smin = m^2 on every leg); else the second, which adds
 * pT 0 / |eta| 99 entries for the internal currents.  smax: the largest
 * number of s-channel joins (the reference's default is 2).  On success *out
 * holds the descriptions in the reference's order (its std::set order, with
 * its rule that descriptions with equal (idx, mass, width) lists are one) and
 * the completed cuts; free with chili_channel_list_free.  err (may be NULL)
 * receives the reason of a failure. */
int chili_construct_channels(double sqrts, const int32_t *flavs, int n_flavs, const chili_model *model,
                             const chili_cuts *cuts, int smax, chili_channel_list **out, char *err, size_t err_len);
/* The list's descriptions and cuts (owned by the list). */
int chili_channel_list_get(const chili_channel_list *list, const chili_channel_desc **descs, int *nch,
                           const chili_cuts **cuts);
void chili_channel_list_free(chili_channel_list *list);

/* Phase-space dimensions of the channels, 3*(n_ext-2)-2 (Channel.hh:33). */
int chili_gpu_ndims(const chili_ctx *ctx);
/* FSMapper::GeneratePoint (Channel.cc:22-38): x[n*ndims] -> mom[n*n_ext*4]
 * (E, px, py, pz per leg).  Host or device. */
int chili_gpu_fsmapper_generate(chili_ctx *ctx, int ch, const double *x,
                                double *mom, int64_t n);
/* FSMapper::GenerateWeight (Channel.cc:40-61): mom -> x_out[n*ndims]
 * (optional), w[n].  Host or device. */
int chili_gpu_fsmapper_weight(chili_ctx *ctx, int ch, const double *mom,
                              double *x_out, double *w, int64_t n);
/* FSMapper::GenerateWeight with the reference's in/out uniform buffer
 * (Channel.cc:40-61, the rans argument): x[n*ndims] is read first and only
 * the entries the channel's inverse map consumes are overwritten, as the
 * reference leaves the rest of its buffer (a t-chain that fails leaves its
 * last entry alone).  Host or device. */
int chili_gpu_fsmapper_weight_inout(chili_ctx *ctx, int ch, const double *mom, double *x, double *w, int64_t n);

/* -------------------------------------------------------- multichannel */
/* Channel weights alpha (MultiChannel.cc:62-67 initialises them to 1/nch). */
int chili_gpu_set_alpha(chili_ctx *ctx, const double *alpha, int nch);
/* Current alpha, best weights and min_diff (MultiChannel.cc:138-154). */
int chili_gpu_get_alpha(chili_ctx *ctx, double *alpha, double *best_alpha,
                        double *min_diff, int nch);
/* Channel selection by the libstdc++ discrete_distribution rule used by
 * Random::SelectIndex (Random.hh:43-45) for uniforms v[n] -> ich[n]. */
int chili_gpu_select_channel(chili_ctx *ctx, const double *v, int32_t *ich,
                             int64_t n);
/* Integrand::GenerateWeight (Integrand.hh:112-123): the combined weight of
 * n points mom[n*n_ext*4] generated in channels ich[n]; optional per-channel
 * densities dens[n*nch] and the chosen channel's inverse x_ich[n*ndims]. */
int chili_gpu_multichannel_weight(chili_ctx *ctx, const double *mom,
                                  const int32_t *ich, double *wgt,
                                  double *dens, double *x_ich, int64_t n);
/* One MultiChannel::operator() (MultiChannel.hh:196-251): points are tried in
 * counter order until params->ncalls are accepted; rejected points count as
 * zero-valued calls.  Uniforms come from the generator (seed, counter_base+k)
 * or, when u is not NULL, from u[k*(ndims+1)...] (ndims uniforms then the
 * channel uniform, MultiChannel.hh:145-147) for k < n_u; running out of u is
 * CHILI_ERR_LIMIT.  Device-resident u is read in place; host u (pinned for
 * asynchronous copies) is uploaded in slices (2^16, 2^18, then 2^19 rows) on a second stream,
 * the rows the last iteration's acceptance rate predicts; each slice is
 * mapped and weighted while the next ones cross PCIe, and rows past the
 * point that completes ncalls are not copied beyond the predicted ones.
 * With should_optimize the channel grids, alpha and best
 * weights are adapted on the device (MultiChannel.hh:182-194).
 * guard_alpha != 0 drops non-finite alpha-training terms, a documented
 * deviation from the reference (which propagates them). */
int chili_gpu_multichannel_iterate(chili_ctx *ctx,
                                   const chili_multichannel_params *params,
                                   uint64_t seed, uint64_t counter_base,
                                   const double *u, int64_t n_u,
                                   int guard_alpha, chili_stats *stats_out,
                                   chili_mc_iter_info *info);
/* Per-channel training histograms [nch*dims*bins] and alpha-training sums
 * [nch] of the last iteration (before adaptation).  Host or device. */
int chili_gpu_get_training(chili_ctx *ctx, double *hist, double *alpha_train);
/* MultiChannel::Train (MultiChannel.hh:182-194) from given training data:
 * channel-weight adaptation (MultiChannel.cc:109-136) from alpha_train [nch],
 * grid adaptation (Integrand.hh:97-104) from hist [nch*dims*bins], best
 * weights (MultiChannel.cc:138-154). With an iteration run at
 * should_optimize = 0 and its own training data this equals the iteration's
 * own training step; with the training data summed over ranks (one
 * all-reduce) it is the reference's MPI mode (MultiChannel.hh:184-190), every
 * rank adapting identically. Host or device. */
int chili_gpu_multichannel_train(chili_ctx *ctx, const chili_multichannel_params *params, const double *hist,
                                 const double *alpha_train);
/* The last iteration's training data and StatsData packed for the MPI
 * mode's exchange (MultiChannel.hh:184-190, MultiChannel.cc:69-77) in one
 * FP64 buffer of len >= nch*dims*bins + nch + 6:
 *   [hist (nch*dims*bins) | alpha_train (nch) | n, sum, sum2, n_finite | max, -min]
 * The first nch*dims*bins + nch + 4 values are summed over the ranks, the
 * last two reduced by maximum; hist and alpha_train of the sums then go to
 * chili_gpu_multichannel_train as device pointers into the same buffer.
 * With a device buffer the copy stays on the device in stream order (no
 * host round trip); host buffers are filled before the call returns. */
int chili_gpu_pack_training(chili_ctx *ctx, double *buf, int64_t len);

/* MultiChannel::SaveAs / LoadFrom (MultiChannel.hh:65-84): the reference's
 * binary results.chili (Integrand::Serialize, then MultiChannel::Serialize)
 * written from / read into this context, so that a grid trained by the
 * reference resumes here and vice versa. Save writes the channel set, grids,
 * params (the 8 serialised fields), best weights, min_diff and the given
 * per-iteration StatsData list. Load checks that the file's channels equal
 * the context's channel set, then sets grids, channel weights = best weights
 * (as the reference's Deserialize does) and min_diff; params (optional)
 * receives the file's params (should_optimize = 1, grid_alpha and iteration
 * kept), results (optional, up to max_results) the StatsData list and
 * nresults (optional) its length. */
int chili_gpu_save_checkpoint(chili_ctx *ctx, const char *path, const chili_multichannel_params *params,
                              const chili_stats *results, int64_t nresults);
int chili_gpu_load_checkpoint(chili_ctx *ctx, const char *path, chili_multichannel_params *params,
                              chili_stats *results, int64_t max_results, int64_t *nresults);

/* Event generation: MultiChannel::GeneratePoint + GenerateWeight
 * (MultiChannel.hh:141-165) for n points in counter order, with no PreProcess
 * and no retry.  mom[n*n_ext*4], wgt[n] = f*w (0 if not finite), ch[n];
 * any output may be NULL.  Host or device. */
int chili_gpu_generate(chili_ctx *ctx, int64_t n, uint64_t seed,
                       uint64_t counter_base, double *mom, double *wgt,
                       int32_t *ch);

/* What one chili_gpu_generate_unweighted call did. */
typedef struct {
    uint64_t points;        /* points drawn (= n)                              */
    uint64_t rejected_pre;  /* PreProcess rejections (value 0, never kept)     */
    uint64_t kept;          /* unweighted events (also those beyond max_events)*/
    uint64_t overweight;    /* kept events with |value| > w_max                */
    double sum;             /* sum of the values of all n points               */
    double max;             /* largest value                                   */
} chili_unweight_info;

/* Unweighted events: the unweighting stage the reference leaves to the
 * PostProcess hook of MultiChannel::operator() (MultiChannel.hh:240-245).
 * n points are drawn in counter order (counters counter_base ...: the same
 * points as chili_gpu_multichannel_iterate draws), passed through PreProcess
 * and given the value v = f * w (the combined multichannel weight; 0 for a
 * rejected point or a NaN value).  Point k is kept when r_k * w_max < |v_k|,
 * r_k the uniform of the "accept" stream (Philox4x32-10, key seed, block
 * {0, lo(k), hi(k), 1}, words 0 and 1).  Kept events are written in counter
 * order: mom[max_events * n_ext * 4], wgt[max_events] = sign(v) max(|v|,
 * w_max) (so that sum(wgt) / n estimates the integral), ch[max_events]; any
 * output may be NULL; n_events (may be NULL) receives the number kept, which
 * counts the events beyond max_events too (they are not written).
 * w_max > 0, e.g. the weight_max of an earlier iteration.  Host or device
 * outputs; no counterpart in the reference's own code. */
int chili_gpu_generate_unweighted(chili_ctx *ctx, int64_t n, uint64_t seed, uint64_t counter_base, double w_max,
                                  double *mom, double *wgt, int32_t *ch, int64_t max_events, int64_t *n_events,
                                  chili_unweight_info *info);

/* Interface::Evaluate (nanobind.hh:23-50) / CallChili (Tensorflow.cc:22-135):
 * uniforms u[n*ndims] through channel ch's FSMapper alone (no VEGAS grid):
 * out[n] = f * FSMapper weight, 0 where PreProcess rejects or the weight is 0.
 * The output buffer is the caller's.  Host or device. */
int chili_gpu_evaluate_batch(chili_ctx *ctx, int ch, const double *u,
                             double *out, int64_t n);

/* ------------------------------------------------ learned proposal */
/* No counterpart in the reference (Chili has no learned proposal): a
 * channel-conditioned rational-quadratic spline coupling flow on each
 * channel's VEGAS uniforms and a softmax channel-weight network, trained
 * online on the GPU (hand-written forward, backward and Adam kernels; bf16
 * tensor-core products with f32 accumulation; f32 splines; FP64 phase space).
 * Estimator per point: v = alpha_c(p) f(p) dens_c(p) J / (beta_c q_c(u)) for
 * the channel c that generated it (c ~ beta, u ~ q_c, x = VEGAS_c(u),
 * p = FSMapper_c(x)). Requires channels (at most 48), grids, integrand and
 * channel weights to be set; beta starts as the current channel weights.
 *
 * Conditioner of layer l, H = hidden units, depth hidden layers:
 * h_1 = lrelu(W1 (2a - 1) + E[c]), h_k = lrelu(W2_{k-2} h_{k-1}) for
 * k = 2..depth, theta = W3 h_depth; unit H-1 of every hidden layer is the
 * constant 1 (it carries the biases).
 * Flat parameter layout (f32): per coupling layer l: W1 [H][da_l],
 * E [nch][H], W2_0 .. W2_{depth-2} [H][H] each, W3 [db_l*49][H]; then the
 * channel-weight network: A1 [64][F], c1 [64], A2 [64][64], c2 [64],
 * A3 [nch][64], c3 [nch], F = n_out(n_out-1)/2 + n_out. Layer l transforms
 * db_l <= 5 dimensions (dims <= 10: alternating, half/half and shifted-pair
 * splits and their complements in turn; dims > 10: dimensions 5l..5l+4 mod
 * dims). */
typedef struct {
    int32_t layers;       /* coupling layers (6) */
    int32_t batch;        /* points per training step (65536) */
    double lr;            /* Adam step size (1e-3) */
    uint64_t init_seed;   /* weight initialisation */
    int32_t hidden;       /* hidden units H of a conditioner: 128 or 256 (0: 128) */
    int32_t depth;        /* hidden layers of a conditioner: 2..4 (0: 2) */
} chili_flow_params;

typedef struct {
    uint64_t points;       /* points drawn */
    uint64_t nonzero;      /* points with v != 0 */
    uint64_t nonfinite;    /* points whose v was not finite (counted as 0) */
    double weight_max;     /* max v */
    double unweighting_efficiency;  /* mean v / max v */
} chili_flow_iter_info;

int chili_gpu_flow_init(chili_ctx *ctx, const chili_flow_params *params);
int64_t chili_gpu_flow_nparams(const chili_ctx *ctx);
/* Flat parameters (layout above). Host or device. */
int chili_gpu_flow_get_params(chili_ctx *ctx, float *prm);
int chili_gpu_flow_set_params(chili_ctx *ctx, const float *prm);
/* Channel-selection probabilities beta [nch] of the flow path. */
int chili_gpu_flow_get_beta(chili_ctx *ctx, double *beta);
int chili_gpu_flow_set_beta(chili_ctx *ctx, const double *beta);
/* Density direction u -> z of the flow of each point's channel, and log q(u);
 * u, z [n][dims] row-major in [0,1]. Host or device. */
int chili_gpu_flow_density(chili_ctx *ctx, const float *u, const int32_t *ch, int64_t n, float *z,
                           float *logq);
/* Sampling direction z -> u, and log q(u). Host or device. */
int chili_gpu_flow_sample_u(chili_ctx *ctx, const float *z, const int32_t *ch, int64_t n, float *u,
                            float *logq);
/* The variance loss mean_i alpha_c^2 F^2 / (beta_c^2 q) on a given batch
 * (u [n][dims], ch [n], logf [n] = log F, -inf for F = 0, feat [n][F],
 * logprior [n][nch]) and its gradient with respect to every parameter
 * (grad [nparams]); no update. Host or device. */
int chili_gpu_flow_loss_grad(chili_ctx *ctx, const float *u, const int32_t *ch, const float *logf,
                             const float *feat, const float *logprior, int64_t n, double *loss, float *grad);
/* `steps` Adam steps, each on a fresh batch drawn from the plain multichannel
 * proposal (counters counter_base + step*batch ...); loss[steps] (host or
 * device, may be NULL) receives each step's loss. */
int chili_gpu_flow_train(chili_ctx *ctx, int steps, uint64_t seed, uint64_t counter_base, double *loss);
/* One integration pass of ncalls points through the flow path (counters
 * counter_base ...); StatsData of v. adapt_beta != 0 sets beta_c proportional
 * to the root mean square of this pass's per-channel terms beta_c v. */
int chili_gpu_flow_iterate(chili_ctx *ctx, uint64_t ncalls, uint64_t seed, uint64_t counter_base,
                           int adapt_beta, chili_stats *stats_out, chili_flow_iter_info *info);
/* Tensor-core check: C[128][N] from f32 A, B rounded to bf16;
 * mode 0: C = A B^T (A [128][K], B [N][K]); mode 1: C = A^T B (A [K][128],
 * B [K][N]); mode 2: C = A B (A [128][K], B [K][N]). K and N multiples of 16
 * in [16, 256]. Host buffers.  Mode 3 checks the failure path: no product is
 * issued, the kernel's bounded wait on its mbarrier gives up (2^16 polls),
 * releases its tensor memory and the call returns CHILI_ERR_TIMEOUT; the
 * context stays usable. */
int chili_gpu_tc_selftest(chili_ctx *ctx, int mode, int K, int N, const float *A, const float *B, float *C);

/* ------------------------------------------------------ batched integrands
 * Many independent integrations advanced together: one persistent launch
 * evaluates the points of every task per iteration, one graph replays the
 * whole iteration (evaluation, per-task StatsData folds, channel-weight
 * updates, grid adaptation).  No counterpart in the reference, which runs one
 * Vegas or MultiChannel object per integrand (Vegas.cc:18-52,
 * MultiChannel.hh:184-260); each task follows that object's algorithm with a
 * fixed budget of ncalls drawn points per iteration: points that PreProcess
 * rejects, or whose value is NaN, count as calls of value 0 (no retries).
 * Task k draws its uniforms from the Philox stream of key seed + k, counter
 * (iteration << 32) + point: a camel task's iteration i equals
 * chili_gpu_vegas_iterate(seed + k, counter_base = i << 32) on the same grid. */
enum chili_task_kind {
    CHILI_TASK_CAMEL = 0,        /* plain VEGAS of the camel (CHILI_FUNC_CAMEL) */
    CHILI_TASK_MULTICHANNEL = 1  /* FSMapper channels + multichannel weights     */
};

typedef struct {
    int32_t kind;           /* chili_task_kind                                  */
    int32_t dims;           /* camel: dimensions (multichannel: from n_ext)      */
    int32_t bins;           /* bins of every grid of the task, [2, MAX_BINS]     */
    uint64_t ncalls;        /* points per iteration, [1, 2^32)                   */
    double grid_alpha;      /* AdaptiveMap::Adapt exponent (VegasParams::alpha)  */
    double beta;            /* MultiChannel::Adapt beta (multichannel)           */
    double min_alpha;       /* MultiChannel::Adapt floor (multichannel)          */
    int32_t fkind;          /* chili_integrand_kind (multichannel)               */
    int32_t nparams;
    const double *params;   /* camel: {s, N, a[dims], b[dims]}                   */
    int32_t pre;            /* chili_preprocess_kind (multichannel)              */
    int32_t nch;            /* channels (multichannel)                           */
    const chili_channel_desc *descs;
    const chili_cuts *cuts;
    double sqrts;
    int32_t n_ext;
    double pre_cuts[4];     /* CHILI_PRE_CUTS: sqrts, ptmin, etamax, delta_r     */
} chili_task;

typedef struct {
    uint32_t block;             /* threads per block of the evaluation launch  */
    uint32_t points_per_thread; /* points per thread per work unit             */
    double ms_per_iteration;    /* device time per iteration of the last call  */
    uint64_t units;             /* work units per iteration                    */
    uint64_t points;            /* calls per iteration, all tasks (ncalls)     */
    uint64_t retry_rounds;      /* retry rounds beyond each iteration's first,
                                   summed over the last call's iterations      */
} chili_batch_info;

/* Replace the context's batch with ntasks tasks (uniform grids, equal channel
 * weights).  Host arrays. */
int chili_gpu_batch_set(chili_ctx *ctx, const chili_task *tasks, int ntasks);
/* `iterations` iterations of every task (adapt != 0: grids and channel
 * weights adapt after each); stats[iterations * ntasks] (host, may be NULL)
 * receives each iteration's StatsData, task-minor.  The first call picks the
 * block size and points per thread by timing the candidates. */
int chili_gpu_batch_iterate(chili_ctx *ctx, int iterations, uint64_t seed, int adapt, chili_stats *stats,
                            chili_batch_info *info);
/* Task `task`'s grids edges[nch * dims * (bins + 1)] and channel weights
 * alpha[nch] (host, either may be NULL). */
int chili_gpu_batch_get_grid(chili_ctx *ctx, int task, double *edges, double *alpha);

#ifdef __cplusplus
}
#endif

#endif /* CHILI_GPU_H */
