"""The FP64 forward-mode replay (oracle/bo_tangent.cpp) that checks the device adjoint:
its directional derivatives against central differences of its own loss, on the CPU.
Also the oracle's release log, which the replay feeds on."""
import numpy as np
import pytest

from bioneuroncore_b200 import (Network, NetgenParams, NET_ADJOINT, NETGEN_FULL_SMALL_SET, NETGEN_GLYCINE,
                                NETGEN_NMDA)

DT = 0.025


def _densities(net):
    seg = net.segments
    N, K = net.data.num_segments, net.data.num_synapses
    out = [np.zeros(N) for _ in range(3)]
    for i in range(N):
        for j in range(seg["modifier_count"][i]):
            c = {141: 0, 142: 0, 123: 1, 107: 2}.get(int(seg["modifiers"][i][j]["type"]))
            if c is not None:
                out[c][i] = float(np.float32(seg["modifiers"][i][j]["density"]))
    return out + [np.ones(K)]


def test_release_log_is_sorted_and_positive():
    from oracle.oracle import Oracle
    p = NetgenParams(family=NET_ADJOINT, n_neurons=4, seed=7)
    syn, tick, amt = Oracle(Network(p)).run_logged(400, DT)
    assert syn.size > 0
    key = syn.astype(np.uint64) * np.uint64(1 << 32) + tick
    assert (np.diff(key.astype(np.float64)) >= 0).all()
    assert (amt > 0).all() and (tick < 400).all()


@pytest.mark.parametrize("flags", [0, NETGEN_FULL_SMALL_SET, NETGEN_GLYCINE, NETGEN_NMDA])
def test_tangent_matches_its_central_differences(flags):
    """With the fitting family, with the whole small set (Cav1.3, the Na/K pump and
    the ATP it consumes, which diffuses), with glycine receptors first on the
    odd-numbered synapses (4 neurons over 400 ticks, where synapse 17, a glycine
    synapse, releases), and with an NMDA receptor after the AMPA one of every
    excitatory synapse (its Ca2+ current, Mg2+ block and Ca2+-dependent inactivation
    gate carry the tangent)."""
    from oracle.oracle import Oracle, tangent_loss
    gly = bool(flags & NETGEN_GLYCINE)
    nmda = bool(flags & NETGEN_NMDA)
    n, ticks = (4, 400) if (gly or nmda) else (3, 300)
    p = NetgenParams(family=NET_ADJOINT, n_neurons=n, seed=7 if (gly or nmda) else 11, flags=flags)
    net = Network(p)
    log = Oracle(Network(p)).run_logged(ticks, DT)
    base = _densities(net)
    soma = np.array([k * 64 for k in range(n)], np.uint32)
    target = np.full((ticks, n), -64.0, np.float32)
    rng = np.random.default_rng(5)
    dvec = [x * rng.standard_normal(x.shape) for x in base]
    zero = [np.zeros_like(x) for x in base]
    if gly:
        is_gly = net.synapses["post_receptors"][:, 0]["type"] == 12
        assert is_gly[np.unique(log[0])].any()          # a glycine synapse releases
    if nmda:
        is_nmda = net.synapses["post_receptors"][:, 1]["type"] == 9
        assert is_nmda[np.unique(log[0])].any()         # an NMDA synapse releases
    dirs = [dvec]
    if gly:   # the weights of the glycine synapses alone
        dirs.append(zero[:3] + [np.where(is_gly, base[3], 0.0)])
    if nmda:  # the weights of the synapses with an NMDA receptor alone
        dirs.append(zero[:3] + [np.where(is_nmda, base[3], 0.0)])
    for dv in dirs:
        L, dL = tangent_loss(net, log, ticks, DT, base, dv, soma, target)
        h = 1e-4
        Lp, _ = tangent_loss(net, log, ticks, DT, [x + h * v for x, v in zip(base, dv)], zero, soma, target)
        Lm, _ = tangent_loss(net, log, ticks, DT, [x - h * v for x, v in zip(base, dv)], zero, soma, target)
        fd = (Lp - Lm) / (2 * h)
        assert L > 0 and abs(dL) > 0
        assert abs(dL - fd) <= 1e-6 * abs(fd), (dL, fd)
