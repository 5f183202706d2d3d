"""CPU tests of the C ABI boundary: the library loads without a GPU, exports
every function the headers in include/ declare, and its host-only entry
points behave (no device work is done here)."""
import ctypes
import os
import re

import numpy as np
import torch

from blastp_b200 import _lib, blosum62, default_params
from blastp_b200 import legacy

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b([A-Za-z_]\w*)\s*\(", text, flags=re.M):
            name = m.group(1)
            if name in ("if", "while", "for", "switch", "return", "sizeof", "defined"):
                continue
            names.add(name)
    return names


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    declared = declared_functions()
    assert {"GPU_BLASTP", "GPU_BLASTP_get_data", "GPU_BLASTP_free_memory", "GPU_BLASTP_check_memory",
            "GPU_BLAST_check_availability", "Round2Multiple", "bp_search", "bp_query_create",
            "bp_db_create"} <= declared
    missing = [n for n in sorted(declared) if not hasattr(L, n)]
    assert not missing, "declared but not exported: %s" % missing
    # and the ctypes signature table covers them all
    assert declared <= set(_lib.SIGNATURES), sorted(declared - set(_lib.SIGNATURES))


def test_library_matrix_equals_reference_fixture(matrix):
    assert (blosum62() == matrix).all()


def test_default_params():
    p = default_params()
    assert (p.word_length, p.threshold, p.window, p.x_dropoff, p.cutoff_score) == (3, 11, 40, 16, 41)


def test_status_strings():
    L = _lib.lib()
    assert L.bp_status_string(0) == b"ok"
    assert L.bp_status_string(7) == b"no CUDA device"


def test_round2multiple_matches_reference_rule():
    # gpu_blastp.c:12-17: round up to a multiple of 64
    for x, want in [(0, 0), (1, 64), (63, 64), (64, 64), (65, 128), (300, 320)]:
        assert legacy.round2multiple(x) == want


def test_no_device_paths_report_cleanly():
    if torch.cuda.is_available():
        return
    L = _lib.lib()
    assert L.GPU_BLAST_check_availability() == 0
    h = ctypes.c_void_p()
    assert L.bp_engine_create(0, ctypes.byref(h)) == 7 and not h.value


def test_gpu_volume_layout_roundtrip():
    # The reference layout (functions.cpp:529-536): residue k of group member i
    # at base + ((k>>2)*G + i)*4 + (k&3).  Check by decoding one subject.
    rng = np.random.default_rng(3)
    lens = np.array([5, 70, 64, 1, 130, 3], dtype=np.int64)
    off = np.concatenate([[0], np.cumsum(lens)])
    res = rng.integers(1, 28, size=int(off[-1])).astype(np.uint8)
    G = 4
    vol, glen, flat, poff = legacy.gpu_volume(res, off, G)
    assert glen.tolist() == [128, 192]
    assert len(vol) == (128 + 192) * G
    for s in range(len(lens)):
        g, i = divmod(s, G)
        base = 0 if g == 0 else 128 * G
        k = np.arange(glen[g])
        got = vol[base + ((k >> 2) * G + i) * 4 + (k & 3)]
        want = np.zeros(glen[g], dtype=np.uint8)
        want[:lens[s]] = res[off[s]:off[s + 1]]
        assert (got == want).all()
        assert (flat[poff[s]:poff[s] + glen[g]] == want).all()


def test_python_mirrors_match_the_header_layouts(tmp_path):
    # every ctypes Structure and record dtype the Python layer passes across the
    # boundary has the size and field offsets the C compiler gives the header's
    # struct of the same name
    from blastp_b200.api import GAPPED_DTYPE, HSP_DTYPE
    mirrors = [("bp_params", _lib.BpParams), ("bp_gapped_params", _lib.BpGappedParams),
               ("bp_batch_options", _lib.BpBatchOptions), ("bp_autotune_trial", _lib.BpAutotuneTrial),
               ("bp_autotune_options", _lib.BpAutotuneOptions), ("bp_server_options", _lib.BpServerOptions),
               ("bp_server_metrics", _lib.BpServerMetrics)]
    dtypes = [("bp_hsp", HSP_DTYPE), ("bp_gapped_hsp", GAPPED_DTYPE)]
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "blastp_b200.h"', 'int main(void) {']
    expect = []
    for cname, cls in mirrors:
        lines.append('printf("%%zu\\n", sizeof(%s));' % cname)
        expect.append(ctypes.sizeof(cls))
        for f in cls._fields_:
            lines.append('printf("%%zu\\n", offsetof(%s, %s));' % (cname, f[0]))
            expect.append(getattr(cls, f[0]).offset)
    for cname, dt in dtypes:
        lines.append('printf("%%zu\\n", sizeof(%s));' % cname)
        expect.append(dt.itemsize)
        for name in dt.names:
            lines.append('printf("%%zu\\n", offsetof(%s, %s));' % (cname, name))
            expect.append(dt.fields[name][1])
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    import subprocess
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    assert got == expect
