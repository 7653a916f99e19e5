"""Generates tests/golden/*.npz from the reference itself: the unmodified Chili
sources compiled into oracle/_ref/libchili_ref.so (oracle/Makefile).

    make -C oracle ref && python tests/golden/make_golden.py

The fixtures pin the C restatement (oracle/port) and the CUDA library on a
machine where the reference sources are absent.  Inputs are seeded; uniforms
are 53-bit (k * 2^-53) so that the reference's generate_canonical reproduces
them exactly.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from chili_b200 import abi, channels, workloads  # noqa: E402
from oracle import ref  # noqa: E402


def random_grid(rng, dims, bins):
    e = np.sort(rng.random((dims, bins - 1)), axis=1)
    return np.concatenate([np.zeros((dims, 1)), e, np.ones((dims, 1))], axis=1)


def grids(rng):
    out = {}
    dims, bins = 4, 50
    e = random_grid(rng, dims, bins)
    u = workloads.uniforms53(rng, (1000, dims))
    u[0] = 0.0
    x, jac = ref.am_map(e, u)
    on_edges = e[:, 1:bins].T.copy()
    xw = np.concatenate([x, on_edges, np.zeros((1, dims)), np.ones((1, dims))])
    w, b = ref.am_weight(e, xw)
    train = rng.random(dims * bins) ** 4
    train[bins:2 * bins] = 0.0
    out.update(grid_edges=e, grid_u=u, grid_x=x, grid_jac=jac, grid_xw=xw, grid_w=w, grid_bin=b,
               grid_train=train, grid_adapted=ref.am_adapt(e, 1.5, train))
    for k in (2, 3, 4):
        out[f"grid_split{k}"] = ref.am_split(e, k)
    p = np.array(workloads.camel_params(dims))
    uv = workloads.uniforms53(rng, (2000, dims))
    st, tr, e2 = ref.vegas_iterate(e, 1.5, p, uv, adapt=True)
    out.update(vegas_params=p, vegas_u=uv, vegas_stats=np.array(st.as_tuple()), vegas_train=tr,
               vegas_edges_after=e2)
    alpha = rng.random(15) ** 3
    alpha[4] = 0.0
    v = workloads.uniforms53(rng, 2000)
    out.update(select_alpha=alpha, select_v=v, select_ich=ref.select(alpha, v))
    return out


def multichannel(rng):
    out = {}
    cs = channels.multichannel_2_to_4()
    params = workloads.mc_params(400)
    R = ref.MultiChannel(cs, 100, params, abi.CHILI_FUNC_PROPAGATOR, channels.propagator_params())
    nd = R.ndims
    xs, moms, ws, xis = [], [], [], []
    for ch in range(cs.nch):
        x = workloads.uniforms53(rng, (100, nd))
        mom = R.fsm_generate(ch, x)
        w, xi = R.fsm_weight(ch, mom)
        xs.append(x), moms.append(mom), ws.append(w), xis.append(xi)
    out.update(fsm_x=np.stack(xs), fsm_mom=np.stack(moms), fsm_w=np.stack(ws), fsm_xinv=np.stack(xis))
    edges = np.stack([random_grid(rng, nd, 100) for _ in range(cs.nch)])
    R.set_grids(edges)
    out["mc_edges0"] = edges
    its = []
    for it in range(3):
        u = workloads.uniforms53(rng, (1600, nd + 1))
        st, info = R.iterate(u, guard=True)
        a, b, md = R.get_alpha()
        h, atr = R.training()
        its.append(dict(u=u, stats=np.array(st.as_tuple()),
                        info=np.array([info.points_tried, info.rejected_pre, info.rejected_nan,
                                       info.weight_max, info.nonfinite_alpha_terms]),
                        alpha=a, best=b, min_diff=np.array([md]), grids=R.get_grids(), hist=h, atrain=atr))
    for k in its[0]:
        if k in ("grids", "hist"):
            out[f"mc_{k}"] = its[-1][k]  # state after the last iteration only
        else:
            out[f"mc_{k}"] = np.stack([d[k] for d in its])
    # combined weight on fixed momenta with the adapted state
    ich = rng.integers(0, cs.nch, 1000).astype(np.int32)
    x = workloads.uniforms53(rng, (1000, nd))
    mom = np.stack([R.fsm_generate(int(c), x[i:i + 1])[0] for i, c in enumerate(ich)])
    ok = ~np.isnan(mom).any(axis=(1, 2))
    mom, ich = mom[ok], ich[ok]
    w, dens, xi = R.weight(mom, ich)
    out.update(cw_mom=mom, cw_ich=ich, cw_w=w, cw_dens=dens, cw_x=xi, cw_alpha=R.get_alpha()[0],
               cw_grids=R.get_grids())
    u = workloads.uniforms53(rng, (300, nd))
    out.update(eval_u=u, eval_out=np.stack([R.evaluate_batch(ch, u) for ch in (0, 7, 12)]))
    return out


def main():
    rng = np.random.default_rng(20261203)
    np.savez_compressed(os.path.join(HERE, "grids.npz"), **grids(rng))
    np.savez_compressed(os.path.join(HERE, "multichannel_2to4.npz"), **multichannel(rng))
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
