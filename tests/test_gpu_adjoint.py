"""The adjoint (bnc_adjoint_*): replay forward against the plain tick, gradients
against central finite differences, and a fit that the gradients drive.

The network is the fitting family (BNC_NET_ADJOINT: Nav1.x, Kv_DR and K2P leak per
segment, myelin on alternate axon segments, Cav2.1 on axons, AMPA/GABA-A synapses,
a 1 nA step into 10% of somata), and for the replay and the gradients also the same
family with the whole small set (BNC_NETGEN_FULL_SMALL_SET: Cav1.3 and the Na/K pump
on every segment, the pump's ATP diffusing), with glycine receptors, and with an NMDA
receptor after the AMPA one of every excitatory synapse (BNC_NETGEN_NMDA: Ca2+ current,
Mg2+ block, Ca2+-dependent inactivation gate).  All tests are marked gpu.
"""
import numpy as np
import pytest

from bioneuroncore_b200 import (Adjoint, Backend, Network, NetgenParams, NET_ADJOINT, NETGEN_FULL_SMALL_SET,
                                NETGEN_GLYCINE, NETGEN_NMDA)

DT = 0.025

pytestmark = pytest.mark.gpu


def _setup(n_neurons, ticks, n_sets, seed=7, checkpoint_every=64, sample_every=1, flags=0):
    p = NetgenParams(family=NET_ADJOINT, n_neurons=n_neurons, seed=seed, flags=flags)
    net = Network(p)
    b = Backend()
    b.load_network(net)
    adj = Adjoint(b, n_sets, ticks, DT, checkpoint_every=checkpoint_every, sample_every=sample_every)
    adj.record()
    return p, net, b, adj


def _plain_soma_trace(p, soma, ticks):
    b = Backend()
    b.load_network(Network(p))
    out = np.zeros((ticks, len(soma)), np.float32)
    for t in range(ticks):
        b.run_ticks(1, DT)
        out[t] = np.asarray(b.segment_field("V", 0), np.float32)[soma]
    return out


@pytest.mark.parametrize("flags", [0, NETGEN_FULL_SMALL_SET, NETGEN_GLYCINE, NETGEN_NMDA])
def test_replay_forward_is_the_plain_trajectory(flags):
    """The forward pass, replaying the release log, reproduces the plain tick's somatic
    voltages bit for bit (same device functions, same operation order)."""
    ticks = 300
    p, net, b, adj = _setup(6, ticks, 2, flags=flags)
    assert adj.release_count() > 0
    _, tr = adj.forward(trace=True)
    plain = _plain_soma_trace(p, adj.soma, ticks)
    for s in range(2):
        same = tr[s].view(np.uint32) == plain.view(np.uint32)
        assert same.all(), "set %d: %d of %d samples differ, max |diff| %g" % (
            s, int((~same).sum()), same.size, float(np.abs(tr[s] - plain).max()))
    # the stimulated soma crosses the spike threshold (-40 mV) within the run
    assert plain.max() > -40.0


def _fit_problem(ticks, n_sets, n_neurons=4, scale=(1.1, 0.9, 1.2, 0.8), flags=0):
    """Targets from a hidden parameter set: the network's densities times `scale`."""
    p, net, b, adj = _setup(n_neurons, ticks, n_sets, checkpoint_every=64, flags=flags)
    base = [x.astype(np.float32) for x in adj.get_params(0)]
    adj.set_params(0, *[x * s for x, s in zip(base, scale)])
    _, tr = adj.forward(trace=True)
    adj.set_params(0, *base)
    adj.set_target(tr[0])
    return p, net, adj, base, tr[0]


@pytest.mark.parametrize("flags", [0, NETGEN_FULL_SMALL_SET, NETGEN_GLYCINE, NETGEN_NMDA])
def test_gradient_matches_fp64_forward_mode_and_central_differences(flags):
    """The device adjoint's gradient along a random direction of all parameters (gNa,
    gK, gleak per segment, weight per synapse) against (a) the FP64 CPU forward-mode
    replay of the same tick (oracle/bo_tangent.cpp) and (b) central differences of that
    FP64 replay's loss with h = 1e-3 relative to each parameter.  Tolerance 1e-3
    relative: the FP32 device trajectory and the FP64 replay differ by ~1e-4 in the
    gradient over 400 ticks.  Central differences of the FP32 device loss itself are
    rounding-limited at this h and are not the reference."""
    from oracle.oracle import Oracle, tangent_loss
    ticks = 400
    p, net, adj, base, target = _fit_problem(ticks, 1, flags=flags)
    _, _ = adj.forward()
    g = adj.backward()
    log = Oracle(Network(p)).run_logged(ticks, DT)
    assert len(log[0]) == adj.release_count() > 0
    rng = np.random.default_rng(3)
    dirs = [rng.standard_normal(x.shape) for x in base]
    b64 = [x.astype(np.float64) for x in base]
    dvec = [x * d for x, d in zip(b64, dirs)]
    ad = sum(float(np.dot(g[k][0].astype(np.float64), dvec[k])) for k in range(4))
    zero = [np.zeros_like(x) for x in b64]
    L0, tan = tangent_loss(Network(p), log, ticks, DT, b64, dvec, adj.soma, target)
    h = 1e-3
    Lp, _ = tangent_loss(Network(p), log, ticks, DT, [x + h * v for x, v in zip(b64, dvec)], zero, adj.soma, target)
    Lm, _ = tangent_loss(Network(p), log, ticks, DT, [x - h * v for x, v in zip(b64, dvec)], zero, adj.soma, target)
    fd = (Lp - Lm) / (2 * h)
    assert abs(tan - fd) <= 1e-6 * abs(fd)            # the FP64 replay's own consistency
    assert abs(ad - tan) <= 1e-3 * abs(tan), "adjoint %.9g vs FP64 forward mode %.9g" % (ad, tan)
    assert abs(ad - fd) <= 1e-3 * abs(fd), "adjoint %.9g vs central differences %.9g" % (ad, fd)
    # each parameter class on its own
    for k in range(4):
        dk = [np.zeros_like(x) for x in b64]
        dk[k] = dvec[k]
        _, tk = tangent_loss(Network(p), log, ticks, DT, b64, dk, adj.soma, target)
        ak = float(np.dot(g[k][0].astype(np.float64), dvec[k]))
        assert abs(ak - tk) <= 1e-2 * abs(tk) + 1e-6, "class %d: adjoint %.9g vs FP64 forward mode %.9g" % (k, ak, tk)
    if flags & NETGEN_NMDA:
        # the weights of the synapses with an NMDA receptor, one of which releases
        is_nmda = net.synapses["post_receptors"][:, 1]["type"] == 9
        assert is_nmda[np.unique(log[0])].any()
        dk = [np.zeros_like(x) for x in b64]
        dk[3] = np.where(is_nmda, dvec[3], 0.0)
        _, tk = tangent_loss(Network(p), log, ticks, DT, b64, dk, adj.soma, target)
        ak = float(np.dot(g[3][0].astype(np.float64), dk[3]))
        assert abs(tk) > 1e-4
        assert abs(ak - tk) <= 1e-2 * abs(tk), "NMDA synapses' weights: adjoint %.9g vs FP64 forward mode %.9g" % (ak, tk)


def test_fit_reduces_the_loss_from_the_untrained_parameters():
    """The learned part: gradient descent (Adam on log-parameters) with the device
    forward/backward pair fits the conductances and weights to targets made by a hidden
    parameter set.  Four parameter sets with different step sizes train side by side in
    one launch; the best ends at a small fraction of the loss of the untrained
    (initial) parameters, which is what the method without the fit delivers."""
    ticks = 400
    n_sets = 4
    p, net, adj, base, target = _fit_problem(ticks, n_sets, scale=(1.15, 0.85, 1.25, 0.8))
    lrs = [0.01, 0.03, 0.06, 0.1]
    mask = [x > 0 for x in base]
    logp = [[np.log(np.where(mk, x, 1.0)) for x, mk in zip(base, mask)] for _ in range(n_sets)]
    m1 = [[np.zeros_like(x) for x in base] for _ in range(n_sets)]
    m2 = [[np.zeros_like(x) for x in base] for _ in range(n_sets)]
    history = []
    for it in range(40):
        prm = [[np.where(mk, np.exp(lp), 0.0).astype(np.float32) for lp, mk in zip(logp[s], mask)]
               for s in range(n_sets)]
        for s in range(n_sets):
            adj.set_params(s, *prm[s])
        loss, _ = adj.forward()
        history.append(loss.copy())
        g = adj.backward()
        for s in range(n_sets):
            for k in range(4):
                gl = g[k][s].astype(np.float64) * prm[s][k]          # d loss / d log(parameter)
                m1[s][k] = 0.9 * m1[s][k] + 0.1 * gl
                m2[s][k] = 0.999 * m2[s][k] + 0.001 * gl * gl
                mh = m1[s][k] / (1 - 0.9 ** (it + 1))
                vh = m2[s][k] / (1 - 0.999 ** (it + 1))
                logp[s][k] = logp[s][k] - lrs[s] * mh / (np.sqrt(vh) + 1e-12) * mask[k]
    history = np.array(history)
    untrained = history[0]
    assert np.allclose(untrained, untrained[0])             # every set starts at the same loss
    best = history[-1].min()
    assert best < 0.1 * untrained[0], "loss %g after training vs %g untrained" % (best, untrained[0])
