"""Every .bion version the reference reads (3-14), read as the reference reads it.

The reference's bion_load_host (src/bion_loader_host.cpp:26-428) migrates older files
by version and, from version 10 on, by the record sizes in the header
(include/bion_format.h:59-340).  Here files of each layout are written byte by byte --
records of random floats, with the fields the loader validates (indices, counts,
types) set in range -- and loaded by the reference's loader and by bnc_bion_load; the
headers, neurons, segments, connections, synapses and nuclei must be equal byte for
byte.  The bytes the reference's migrations leave unwritten (heap memory from new[]:
a v3-v6 synapse past its 824 bytes, a v3-v8 connection's reserved bytes, a v6 nucleus
past its 332 bytes) are not compared; this library writes zeros there.  For the v3-v6
synapse case the network holds enough synapses that the reference's array is fresh
(zeroed) memory, since its validation reads post_receptor_count from those bytes.
Error codes for malformed files must match too.
"""
import ctypes as C

import numpy as np
import pytest

from oracle.oracle import reference_available, REF_LIB

pytestmark = pytest.mark.skipif(not reference_available(), reason="reference CPU library not built here")

N_SEG = 40
N_NEURON = 8

# segment record size -> offset of modifier_count and its bound (the v3 and v4-v6
# records hold 16 modifiers)
SEG_COUNT = {852: (768, 16), 1692: (1604, 16), 1696: (1604, 32), 1704: (1612, 32), 3208: (3112, 32),
             3216: (3112, 32)}
# synapse record size -> offsets of the pre / post receptor counts the validation reads
SYN_COUNTS = {824: (736,), 836: (384, 740), 1560: (736, 1444), 1568: (736, 1448), 840: (736,), 844: (736,)}


def _ref():
    ref = C.CDLL(REF_LIB)
    load = getattr(ref, "_Z14bion_load_hostPKcP8BionData")
    load.argtypes = [C.c_char_p, C.c_void_p]
    load.restype = C.c_int
    unload = getattr(ref, "_Z16bion_unload_hostP8BionData")
    unload.argtypes = [C.c_void_p]
    return load, unload


def _floats(rng, nbytes):
    n = (nbytes + 3) // 4
    return bytearray(rng.uniform(-50.0, 50.0, n).astype(np.float32).tobytes()[:nbytes])


def _u32(buf, off, v):
    buf[off:off + 4] = np.uint32(v).tobytes()


def _file(path, version, seg_sz, syn_sz, n_syn, conn_sz, nuc_sz=0, n_nuc=0, file_sizes=None, seed=0,
          fix=None):
    """Writes a .bion of `version` with records of the given sizes; returns its bytes."""
    rng = np.random.default_rng(seed)
    hdr_sz = 68 if version < 5 else (84 if version < 10 else 100)
    hdr = bytearray(100)
    _u32(hdr, 0, 0x42494F4E)
    _u32(hdr, 4, version)
    for off, v in ((12, N_NEURON), (16, N_SEG), (20, N_SEG - 1), (24, n_syn)):
        _u32(hdr, off, v)
    hdr[44:68] = _floats(rng, 24)   # timestamp and build id: carried as they are
    if version >= 5:
        _u32(hdr, 68, n_nuc)
        _u32(hdr, 72, 1)
    if version >= 10:
        for off, v in zip(range(76, 100, 4), file_sizes or (seg_sz, syn_sz, nuc_sz or 500, 16, 24, 88)):
            _u32(hdr, off, v)
    out = bytearray(hdr[:hdr_sz])
    for i in range(N_NEURON):   # id, segment_start, segment_count, soma, threshold, type
        rec = _floats(rng, 24)
        _u32(rec, 0, 100 + i)
        _u32(rec, 4, i * (N_SEG // N_NEURON))
        _u32(rec, 8, N_SEG // N_NEURON)
        out += rec
    off_c, bound = SEG_COUNT.get(seg_sz, (None, None))
    for i in range(N_SEG):
        rec = _floats(rng, seg_sz)
        if off_c is not None:
            rec[off_c] = int(rng.integers(0, bound + 1))
        out += rec
    for i in range(N_SEG - 1):   # a chain
        rec = _floats(rng, conn_sz)
        _u32(rec, 0, i)
        _u32(rec, 4, i + 1)
        if conn_sz == 12 and i % 3 == 0:
            rec[8:12] = np.float32(0.0).tobytes()   # no coupling: not intracellular
        if conn_sz == 16:
            rec[8] = i % 2
        out += rec
    for i in range(n_syn):
        rec = _floats(rng, syn_sz)
        _u32(rec, 4, int(rng.integers(0, N_SEG)))
        _u32(rec, 8, int(rng.integers(0, N_SEG)))
        rec[12] = int(rng.integers(0, 3))
        for off in SYN_COUNTS.get(syn_sz, ()):
            rec[off] = int(rng.integers(0, 9))
        out += rec
    for i in range(n_nuc):
        out += _floats(rng, nuc_sz)
    if fix:
        fix(out, hdr_sz)
    path.write_bytes(bytes(out))
    return out


def _bytes(ptr, n):
    return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_uint8)), (n,)).copy() if n else np.zeros(0, np.uint8)


def _mask(n_rec, rec_sz, undefined):
    """Per-byte mask of the defined bytes of n_rec records: False on [a, b) ranges."""
    m = np.ones((n_rec, rec_sz), bool)
    for a, b in undefined:
        m[:, a:b] = False
    return m.reshape(-1)


def _compare(path, syn_undefined=(), conn_undefined=(), nuc_undefined=()):
    from bioneuroncore_b200 import load_library
    from bioneuroncore_b200.abi import BionData
    load, unload = _ref()
    lib = load_library()
    r, o = BionData(), BionData()
    rc_r = load(str(path).encode(), C.byref(r))
    rc_o = lib.bnc_bion_load(str(path).encode(), C.byref(o))
    try:
        assert rc_o == rc_r, "return code %d, the reference's %d" % (rc_o, rc_r)
        if rc_r != 0:
            return rc_r
        for f in ("num_neurons", "num_segments", "num_connections", "num_synapses", "num_nuclei"):
            assert getattr(o, f) == getattr(r, f), f
        assert bytes(o.header) == bytes(r.header)
        parts = (("neurons", 24, ()), ("segments", 3216, ()), ("connections", 16, conn_undefined),
                 ("synapses", 1568, syn_undefined), ("nuclei", 500, nuc_undefined))
        counts = {"neurons": r.num_neurons, "segments": r.num_segments, "connections": r.num_connections,
                  "synapses": r.num_synapses, "nuclei": r.num_nuclei}
        for name, sz, undef in parts:
            n = counts[name]
            a = _bytes(getattr(o, name), n * sz)
            b = _bytes(getattr(r, name), n * sz)
            m = _mask(n, sz, undef)
            bad = np.flatnonzero((a != b) & m)
            assert bad.size == 0, "%s: %d bytes differ, first at record %d byte %d" % (
                name, bad.size, bad[0] // sz, bad[0] % sz)
        return 0
    finally:
        if rc_r == 0:
            unload(C.byref(r))
        if rc_o == 0:
            lib.bnc_bion_unload(C.byref(o))


CONN12_UNDEF = [(9, 12)]                   # reserved bytes a v3-v8 connection never sets
SYN6_UNDEF = [(824, 1540), (1552, 1568)]   # past the 824 copied bytes, except the pool fields
NUC6_UNDEF = [(332, 388), (428, 500)]      # past the 332 copied bytes, except genes 36-45


def test_v3(tmp_path):
    _file(tmp_path / "v3.bion", 3, 852, 824, 0, 12)
    assert _compare(tmp_path / "v3.bion", conn_undefined=CONN12_UNDEF) == 0


def test_v4(tmp_path):
    _file(tmp_path / "v4.bion", 4, 1692, 824, 0, 12, seed=1)
    assert _compare(tmp_path / "v4.bion", conn_undefined=CONN12_UNDEF) == 0


def test_v5_nuclei_of_20_genes(tmp_path):
    _file(tmp_path / "v5.bion", 5, 1692, 824, 0, 12, nuc_sz=204, n_nuc=6, seed=2)
    assert _compare(tmp_path / "v5.bion", conn_undefined=CONN12_UNDEF) == 0


def test_v6_synapses_without_pools_and_nuclei_of_36_genes(tmp_path):
    # 26,000 synapses: the reference's new[] of 40.8 MB is a fresh mapping (zeroed), so
    # its validation of post_receptor_count, which it reads from unwritten bytes, passes
    _file(tmp_path / "v6.bion", 6, 1692, 824, 26000, 12, nuc_sz=332, n_nuc=5, seed=3)
    assert _compare(tmp_path / "v6.bion", syn_undefined=SYN6_UNDEF, conn_undefined=CONN12_UNDEF,
             nuc_undefined=NUC6_UNDEF) == 0


@pytest.mark.parametrize("version,conn_sz", [(7, 12), (8, 12), (9, 16)])
def test_v7_to_v9(tmp_path, version, conn_sz):
    p = tmp_path / ("v%d.bion" % version)
    _file(p, version, 1692, 836, 60, conn_sz, nuc_sz=500, n_nuc=4, seed=version)
    assert _compare(p, conn_undefined=CONN12_UNDEF if conn_sz == 12 else ()) == 0


@pytest.mark.parametrize("seg_sz,syn_sz,nuc_sz", [(1692, 836, 412), (1696, 836, 412), (1704, 844, 500),
                                                  (1800, 840, 500), (3208, 1560, 500), (3216, 1568, 412)])
def test_v10_to_v13_by_record_size(tmp_path, seg_sz, syn_sz, nuc_sz):
    p = tmp_path / "v10.bion"
    version = 13 if seg_sz == 3208 else (12 if seg_sz == 1800 else 10)
    _file(p, version, seg_sz, syn_sz, 50, 16, nuc_sz=nuc_sz, n_nuc=3, seed=seg_sz)
    assert _compare(p) == 0


def test_v14_without_nuclei_gets_default_nuclei(tmp_path):
    p = tmp_path / "v14.bion"
    _file(p, 14, 3216, 1568, 30, 16, seed=14)
    assert _compare(p) == 0
    from bioneuroncore_b200 import load_library
    from bioneuroncore_b200.abi import BionData
    d = BionData()
    assert load_library().bnc_bion_load(str(p).encode(), C.byref(d)) == 0
    try:
        nu = _bytes(d.nuclei, d.num_nuclei * 500).reshape(-1, 500)
        assert d.num_nuclei == N_NEURON
        assert np.array_equal(nu[:, :4].copy().view(np.uint32).ravel(), 100 + np.arange(N_NEURON))
        assert (nu[:, 4] == 1).all() and (nu[:, 5] == 3).all()
        assert np.array_equal(nu[:, 492:496].copy().view(np.float32).ravel(), np.full(N_NEURON, 0.5, np.float32))
    finally:
        load_library().bnc_bion_unload(C.byref(d))


def _set_u32(at):
    def fix(buf, hdr_sz):
        off, v = at(hdr_sz)
        _u32(buf, off, v)
    return fix


@pytest.mark.parametrize("case", ["magic", "version2", "version15", "zero_segments", "short", "connection",
                                  "synapse_type", "modifier_count", "neuron_range"])
def test_malformed_files_fail_as_the_reference_fails(tmp_path, case):
    p = tmp_path / (case + ".bion")
    # version 9 layouts; version 14 for the modifier count, which 9's migration clamps
    seg_sz = 3216 if case == "modifier_count" else 1692
    spec = dict(version=14 if case == "modifier_count" else 9, seg_sz=seg_sz,
                syn_sz=1568 if case == "modifier_count" else 836, n_syn=10, conn_sz=16, seed=7)
    seg0 = lambda h: h + N_NEURON * 24                         # noqa: E731
    conn0 = lambda h: seg0(h) + N_SEG * seg_sz                 # noqa: E731
    syn0 = lambda h: conn0(h) + (N_SEG - 1) * 16               # noqa: E731
    fix = {
        "magic": _set_u32(lambda h: (0, 0x12345678)),
        "version2": _set_u32(lambda h: (4, 2)),
        "version15": _set_u32(lambda h: (4, 15)),
        "zero_segments": _set_u32(lambda h: (16, 0)),
        "connection": _set_u32(lambda h: (conn0(h) + 16 * 5 + 4, N_SEG)),
        "modifier_count": lambda b, h: b.__setitem__(seg0(h) + 3216 * 3 + 3112, 40),
        "neuron_range": _set_u32(lambda h: (h + 24 * 2 + 8, N_SEG)),
        "synapse_type": lambda b, h: b.__setitem__(syn0(h) + 836 * 4 + 12, 3),
    }.get(case)
    data = _file(p, fix=fix, **spec)
    if case == "short":
        p.write_bytes(bytes(data[:-500]))
    rc = _compare(p)
    assert rc < 0
