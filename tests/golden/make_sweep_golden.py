"""Generates the parameter-sweep fixture in this folder from the reference's own CPU tick.

Each task follows the reference's batch mode (daemon_main.cpp:160-300): the
parameter overrides set state[0] of each segment's first modifier of the type
(daemon_main.cpp:79-155), the seed scales every synapse's release probability
(daemon_main.cpp:199-206), and the loop increments the tick counter once more after
each core_run_tick (daemon_main.cpp:250-258), at dt = 0.1 ms.  The overrides and the
seed are applied here in Python, independently of the library; the ticks and the
metrics (core_compute_metrics, simulation_host.cpp:825-880) are the reference's, from
oracle/_ref/libbiocore_ref.so.

    python tests/golden/make_sweep_golden.py
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

DT = 0.1
TICKS = 300
# 3 nA steps of 10 ms: under the batch mode's doubled tick counter they end after
# 50 ticks instead of 100
SPEC = dict(family=1, n_neurons=8, seed=7, stim_pA=3000.0, stim_duration_ms=10.0)
TASKS = [
    ([], 0),
    ([(107, 50.0)], 11),
    ([(141, 0.3), (123, 0.2)], 12345),
]


def apply_task(net, overrides, seed):
    """The reference's overrides and seed variation on a Network's AoS, in place."""
    seg = net.segments
    for tid, val in overrides:
        for i in range(net.data.num_segments):
            types = seg["modifiers"][i]["type"]
            for j in range(types.size):
                if types[j] == tid and types[j] != 0:
                    seg["modifiers"][i][j]["state"][0] = np.float32(val)
                    break
    if seed:
        syn = net.synapses
        for k in range(net.data.num_synapses):
            h = (int(seed) ^ ((int(syn["id"][k]) * 2654435761) & 0xFFFFFFFF)) & 0xFFFFFFFF
            var = np.float32(np.float32(h & 0xFFFF) / np.float32(65536.0)) * np.float32(0.02)
            syn["release_probability"][k] = np.float32(syn["release_probability"][k] * np.float32(1.0 + var))


def run_reference_task(overrides, seed):
    from bioneuroncore_b200 import Network, NetgenParams
    from oracle.oracle import Reference, reference_lib
    net = Network(NetgenParams(**SPEC))
    apply_task(net, overrides, seed)
    ref = Reference(net)
    lib = reference_lib()
    spikes = np.zeros(net.data.num_segments, np.uint32)
    lib.core_enable_spike_count(spikes.ctypes.data, net.data.num_segments)
    ref.run(TICKS, DT, tick_stride=2)
    lib.core_disable_spike_tracking()
    buf = C.create_string_buffer(2048)
    lib.core_compute_metrics.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_uint64, C.c_char_p,
                                         C.c_size_t]
    lib.core_compute_metrics(net.data.segments, net.data.num_segments, net.data.neurons, net.data.num_neurons,
                             ref.tick.value, buf, 2048)
    return net.segments["V_m"].copy(), spikes.copy(), int(ref.tick.value), buf.value.decode()


def main():
    from oracle.oracle import reference_available
    if not reference_available():
        raise SystemExit("oracle/_ref/libbiocore_ref.so is not built (make -C oracle)")
    out = {"ticks": np.int64(TICKS), "dt": np.float32(DT)}
    out.update({"param_" + k: np.float64(v) for k, v in SPEC.items()})
    for q, (ov, seed) in enumerate(TASKS):
        V, spikes, tick, metrics = run_reference_task(ov, seed)
        out["task%d_V" % q] = V
        out["task%d_spikes" % q] = spikes
        out["task%d_tick" % q] = np.int64(tick)
        out["task%d_metrics" % q] = np.array(metrics)
        out["task%d_overrides" % q] = np.array(ov, np.float64).reshape(-1, 2)
        out["task%d_seed" % q] = np.int64(seed)
        print("task", q, "tick", tick, metrics)
    np.savez_compressed(os.path.join(HERE, "sweep", "small_n8_s7_batch.npz"), **out)
    print("wrote sweep/small_n8_s7_batch.npz")


if __name__ == "__main__":
    main()
