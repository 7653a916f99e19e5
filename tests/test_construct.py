"""ConstructChannels (src/Channel/ChannelNode.cc:74-291) in the library
(chili_construct_channels, host code) against the reference's own
ConstructChannels compiled in oracle/_ref, for several models, processes and
s-channel limits: the same descriptions in the same order (ParticleInfo
(idx, pid, mass, width) lists and decay maps, exactly), and with given cuts
the same completed pT / eta tables.  Runs on the CPU."""
import pytest

from chili_b200 import channels, gpu
from oracle import ref

MZ, GZ = channels.MZ, channels.GZ


def gluon_model():
    return {(21, 21): [21]}, {21: 0.0}, {21: 0.0}


def qcd_model():
    rules = {(21, 21): [21]}
    for q in (1, 2):
        for a, b in ((q, -q), (-q, q)):
            rules[(a, b)] = [21]
        for f in (q, -q):
            rules[(f, 21)] = [f]
            rules[(21, f)] = [f]
    return rules, {1: 0.0, 2: 0.0, 21: 0.0}, {1: 0.0, 2: 0.0, 21: 0.0}


def ew_model():
    """Fermions couple to a photon and a Z; quarks to a gluon."""
    rules = {}

    def add(a, b, out):
        rules.setdefault((a, b), [])
        rules[(a, b)] += out

    for f in (1, 11, 13):
        bosons = [22, 23] + ([21] if f == 1 else [])
        for a, b in ((f, -f), (-f, f)):
            add(a, b, bosons)
        for v in bosons:
            for x in (f, -f):
                add(x, v, [x])
                add(v, x, [x])
    masses = {1: 0.0, 11: 0.0, 13: 0.0, 21: 0.0, 22: 0.0, 23: MZ}
    widths = {1: 0.0, 11: 0.0, 13: 0.0, 21: 0.0, 22: 0.0, 23: GZ}
    return rules, masses, widths


def top_model():
    rules = {(6, -6): [21], (-6, 6): [21], (21, 21): [21], (6, 21): [6], (21, 6): [6], (-6, 21): [-6],
             (21, -6): [-6]}
    return rules, {6: 173.0, 21: 0.0}, {6: 1.4, 21: 0.0}


def as_tuples(cs):
    out = []
    for info, dec in cs.channels:
        t = lambda p: (p.idx, p.pid, p.mass, p.width)
        out.append(([t(p) for p in info], [(t(d.parent), t(d.child1), t(d.child2)) for d in dec]))
    return out


CASES = [
    ("gluon 2->2", gluon_model, [21, 21, 21, 21], (0, 1, 2)),
    ("gluon 2->3", gluon_model, [21, 21, 21, 21, 21], (0, 1, 2)),
    ("gluon 2->4", gluon_model, [21] * 6, (1, 2)),
    ("qcd 2->3", qcd_model, [1, -1, 2, -2, 21], (1, 2)),
    ("ew 2->4", ew_model, [1, -1, 11, -11, 13, -13], (1, 2)),
    ("ew 2->3", ew_model, [11, -11, 13, -13, 22], (2,)),
    ("top 2->3", top_model, [21, 21, 6, -6, 21], (1, 2)),
]


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("name,model,flavs,smaxes", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("with_cuts", [False, True])
def test_construct_channels_matches_the_reference(name, model, flavs, smaxes, with_cuts):
    rules, masses, widths = model()
    for smax in smaxes:
        cuts = channels.default_cuts(flavs, masses, ptmin=25.0, etamax=4.5) if with_cuts else None
        want, ptmin, etamax = ref.construct_channels(1000.0, flavs, rules, masses, widths, cuts=cuts, smax=smax)
        cs = gpu.construct_channels(flavs, rules, masses, widths, 1000.0, cuts=cuts, smax=smax)
        got = as_tuples(cs)
        assert got == [(list(i), list(d)) for i, d in want], (name, smax)
        if with_cuts:
            assert cs_cuts(cs, "ptmin") == ptmin and cs_cuts(cs, "etamax") == etamax
        if smax == max(smaxes):
            assert len(got) > 0, name


def cs_cuts(cs, key):
    c = cs.cuts
    n = getattr(c, "n_" + key)
    arr = getattr(c, key)
    return {arr[k].idx: arr[k].value for k in range(n)}


def test_construct_channels_feeds_the_channel_check():
    """The constructed set passes the library's host-side channel check
    (every description consumes 3 n_out - 4 + 2 uniforms, every current has
    its cut entries)."""
    rules, masses, widths = ew_model()
    cs = gpu.construct_channels([1, -1, 11, -11, 13, -13], rules, masses, widths, 1000.0)
    assert cs.nch > 0
    assert gpu.check_channels(cs) == ""


def test_construct_channels_errors():
    rules, masses, widths = gluon_model()
    with pytest.raises(gpu.ChiliError, match="no mass"):
        gpu.construct_channels([21, 21, 21, 1], rules, masses, widths, 1000.0)
    with pytest.raises(gpu.ChiliError):
        gpu.construct_channels([21, 21], rules, masses, widths, 1000.0)
    with pytest.raises(gpu.ChiliError):
        gpu.construct_channels([21, 21, 21, 21], lambda a, b: 1 / 0, masses, widths, 1000.0)
