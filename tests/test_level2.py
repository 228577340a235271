"""Level II (Archive II) output: byte-identical to the reference's own writer on the same volume.

The fixture tests/golden/level2_volume.npz holds a synthetic volume (the /api/volume header and payload) and the
bytes l2writer.encode_volume (l2writer.py:161-182) made from it (tests/golden/make_level2_volume.py). The CPU test
assembles the radials with the oracle's restatement; the GPU test assembles them with the CUDA kernel from a radar
volume in device memory (ob_radar_write + ob_radar_level2). Both are framed by outbreaklab_b200/level2.py."""
import json
import os

import numpy as np
import pytest

from outbreaklab_b200 import level2 as L2

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "level2_volume.npz")


def _golden():
    z = np.load(GOLD)
    return json.loads(z["header"].tobytes().decode()), z["payload"].tobytes(), z["archive"].tobytes()


def test_host_framing_and_templates_match_reference_bytes():
    from oracle import level2_oracle as LO
    header, payload, archive = _golden()
    recs = L2.records_of(header, LO.radials(header, payload))
    out = L2.frame(header["icao"], header["epoch_ms"], recs)
    assert len(out) == len(archive)
    assert out == archive


def test_metadata_record_layout():
    header, _, _ = _golden()
    tilts = [{"angle": s["angle"], "superRes": s["superRes"], "kind": s["kind"]} for s in header["sweeps"]]
    meta = L2.metadata(tilts, header["epoch_ms"], header["vcp"])
    assert len(meta) == 134 * L2.SEGMENT
    assert meta[131 * L2.SEGMENT + 15] == 3 and meta[132 * L2.SEGMENT + 15] == 5 and meta[133 * L2.SEGMENT + 15] == 2


@pytest.mark.gpu
def test_gpu_radial_assembly_matches_reference_bytes(native):
    import ctypes as C
    from outbreaklab_b200 import _native as N, model as M, workloads as W
    header, payload, archive = _golden()
    g, _ = M.setup_case(W.case_small())
    h = C.c_void_p()
    size = (len(payload) + 3) // 4 * 4
    N.check(N.lib().ob_radar_create(g.h, size, 1192, C.byref(h)))
    try:
        buf = np.frombuffer(payload, np.uint8)
        N.check(N.lib().ob_radar_write(h, buf.ctypes.data, buf.nbytes))
        out = L2.encode_volume_gpu(h, header)
        assert out == archive
        # the records themselves, before compression, equal the restatement's
        from oracle import level2_oracle as LO
        tpl, descs, total = L2.plan(header)
        arr = (L2.ObL2Sweep * len(descs))(*descs)
        raw = np.empty(total, np.uint8)
        t = np.frombuffer(tpl, np.uint8)
        N.check(N.lib().ob_radar_level2(h, arr, len(descs), t.ctypes.data, t.nbytes, raw.ctypes.data, raw.nbytes))
        assert raw.tobytes() == LO.radials(header, payload)
    finally:
        N.lib().ob_radar_destroy(h)
