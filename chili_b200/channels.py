"""Channel descriptions and cut tables for the benchmark workloads.

Chili's ConstructChannels (src/Channel/ChannelNode.cc:69-291) derives channels
from a Model's Combinable callback; the workloads below instead hand-build
their ChannelDescriptions and hand them to the public FSMapper constructor
(include/Channel/Channel.hh:18), as the reference permits.  The same tables
feed the CUDA library and both CPU oracles.

Conventions (ChannelNode.cc:83-93): leg i has idx 1<<i, legs 0 and 1 are the
incoming partons; compound currents carry the OR of their legs' bits.
"""
from itertools import combinations

from .abi import ChannelSet, Decay, ParticleInfo

MZ = 91.1876
GZ = 2.4952
PID_Z = 23
PID_MASSLESS = 22


def default_cuts(flavs, masses=None, ptmin=30.0, etamax=99.0, delta_r=0.4):
    """The cut tables ConstructChannels fills by default (ChannelNode.cc:69-95):
    deltaR 0.4 between all flavour pairs (0 if either is a top), and per leg
    smin = m^2, ptmin = 30, etamax = 99; sexternal = m^2 of the outgoing legs."""
    masses = masses or {}
    cuts = {"sexternal": [], "deltaR": {}, "smin": {}, "ptmin": {}, "etamax": {}}
    for f1 in flavs:
        for f2 in flavs:
            cuts["deltaR"][(f1, f2)] = 0.0 if (abs(f1) == 6 or abs(f2) == 6) else delta_r
    for i, f in enumerate(flavs):
        m = masses.get(abs(f), 0.0)
        cuts["smin"][1 << i] = m * m
        cuts["ptmin"][1 << i] = ptmin
        cuts["etamax"][1 << i] = etamax
        if i > 1:
            cuts["sexternal"].append(m * m)
    return cuts


def _add_current(cuts, idx):
    # compound currents: ptmin 0, etamax 99 (ChannelNode.cc:161-162)
    cuts["ptmin"].setdefault(idx, 0.0)
    cuts["etamax"].setdefault(idx, 99.0)


def _leg(flavs, i):
    return ParticleInfo(1 << i, flavs[i], 0.0, 0.0)


def _pair_decay(flavs, i, j, pid, mass, width):
    a, b = _leg(flavs, i), _leg(flavs, j)
    parent = ParticleInfo((1 << i) | (1 << j), pid, mass, width)
    return parent, Decay(parent, a, b)   # children ordered by idx (ChannelNode.cc:175)


def _sorted_desc(infos):
    # ConstructChannels keeps info sorted by std::greater (ChannelNode.cc:221)
    return sorted(infos, key=lambda p: p.key(), reverse=True)


def pair_channel(flavs, pairs, pid, mass, width, cuts):
    """Channel whose t-chain holds the given pair currents (each decaying to
    its two legs) and the remaining outgoing legs, in canonical order."""
    n = len(flavs)
    used = set()
    info, decays = [], []
    for (i, j) in pairs:
        parent, dec = _pair_decay(flavs, i, j, pid, mass, width)
        info.append(parent)
        decays.append(dec)
        used |= {i, j}
        _add_current(cuts, parent.idx)
    info += [_leg(flavs, k) for k in range(2, n) if k not in used]
    return _sorted_desc(info), decays


def t_channel(flavs, last):
    """Pure multi-peripheral chain with leg `last` balancing momentum
    (GenTChan, Channel.cc:115-158: the last info entry is special)."""
    n = len(flavs)
    others = _sorted_desc([_leg(flavs, k) for k in range(2, n) if k != last])
    return others + [_leg(flavs, last)], []


def process_2_to_n(n_out):
    """Flavours of a 2 -> n_out process: q qbar -> alternating lepton pairs."""
    out = []
    for k in range(n_out):
        out.append((11 + 2 * (k // 2)) * (1 if k % 2 == 0 else -1))
    return [1, -1] + out


def multichannel_2_to_4(sqrts=1000.0):
    """The 2->4 workload: 15 channels = 6 s-channel (one Z -> pair per
    outgoing pair, Breit-Wigner sampling) + 9 t-channel (3 pure
    multi-peripheral chains with legs 2, 3, 4 balancing momentum, and 6 chains
    with one massless pair current sampled as s^-0.99)."""
    flavs = process_2_to_n(4)
    cuts = default_cuts(flavs)
    pairs = list(combinations(range(2, 6), 2))
    channels = [pair_channel(flavs, [p], PID_Z, MZ, GZ, cuts) for p in pairs]
    channels += [t_channel(flavs, last) for last in (2, 3, 4)]
    channels += [pair_channel(flavs, [p], PID_MASSLESS, 0.0, 0.0, cuts) for p in pairs]
    return ChannelSet(channels, cuts, sqrts, len(flavs))


def multichannel_2_to_6(sqrts=1000.0):
    """The 2->6 workload: 45 channels = 15 s-channel (Z -> pair for every
    outgoing pair) + 30 t-channel (15 single massless pair currents, 6 pure
    chains with each outgoing leg balancing momentum, 9 chains with two
    disjoint massless pair currents)."""
    flavs = process_2_to_n(6)
    cuts = default_cuts(flavs)
    legs = range(2, 8)
    pairs = list(combinations(legs, 2))
    channels = [pair_channel(flavs, [p], PID_Z, MZ, GZ, cuts) for p in pairs]
    channels += [pair_channel(flavs, [p], PID_MASSLESS, 0.0, 0.0, cuts) for p in pairs]
    channels += [t_channel(flavs, last) for last in legs]
    doubles = [((2, 3), (4, 5)), ((2, 3), (6, 7)), ((4, 5), (6, 7)),
               ((2, 4), (3, 5)), ((2, 4), (6, 7)), ((3, 5), (6, 7)),
               ((2, 5), (3, 4)), ((2, 5), (6, 7)), ((3, 4), (6, 7))]
    channels += [pair_channel(flavs, list(d), PID_MASSLESS, 0.0, 0.0, cuts) for d in doubles]
    return ChannelSet(channels, cuts, sqrts, len(flavs))


def multichannel_2_to_n(n_out, sqrts):
    """A 2->n_out propagator workload (n_out = 2..5): one Z -> pair channel per
    outgoing pair and one pure multi-peripheral chain per outgoing leg."""
    flavs = process_2_to_n(n_out)
    cuts = default_cuts(flavs)
    legs = range(2, 2 + n_out)
    channels = []
    if n_out >= 2:
        for p in combinations(legs, 2):
            if n_out == 2:
                continue  # a 2->2 pair current would be the whole final state
            channels.append(pair_channel(flavs, [p], PID_Z, MZ, GZ, cuts))
    channels += [t_channel(flavs, last) for last in legs]
    return ChannelSet(channels, cuts, sqrts, len(flavs))


def propagator_params(mass=MZ, width=GZ, mt=10.0):
    """Integrand parameters {M, G, m} of CHILI_FUNC_PROPAGATOR(_TOP2)."""
    return [mass, width, mt]
