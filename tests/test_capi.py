"""CPU-side checks of the C ABI: libits.so loads and exports every function that
include/its/its.h declares (no compute call, no GPU needed)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "its", "its.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:its_status|const char\*|int64_t)\s+(its_\w+)\s*\(", src, flags=re.M)))


def test_header_declares_api():
    names = declared_functions()
    assert "its_svo_build" in names and "its_lscg_solve" in names and len(names) > 25


def test_library_exports_every_declared_symbol():
    from its_b200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_host_preprocessing_matches_oracle():
    import numpy as np
    import oracle
    from its_b200 import api, meshes
    V, F = meshes.config_mesh("c0")
    a, b = api.model_to_unit_cube(V), oracle.model_to_unit_cube(V)
    assert np.array_equal(a, b)
    for x, y in zip(api.uniform_bbox(a), oracle.uniform_bbox(b)):
        assert np.array_equal(x, y)


def test_ctypes_structs_match_the_header(tmp_path):
    # the Python binding's structs have the C layout of include/its/its.h (sizes and offsets)
    import subprocess
    from its_b200 import _lib
    src = tmp_path / "sizes.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "its/its.h"\n'
                   'int main(void) { printf("%zu %zu %zu %zu %zu %zu\\n", sizeof(its_svo_info), '
                   'offsetof(its_svo_info, learned_tables_ms), sizeof(its_solve_opts), sizeof(its_solve_report), '
                   'sizeof(its_basis_opts), offsetof(its_basis_opts, num_samples)); return 0; }\n')
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [ctypes.sizeof(_lib.SvoInfo), _lib.SvoInfo.learned_tables_ms.offset, ctypes.sizeof(_lib.SolveOpts),
            ctypes.sizeof(_lib.SolveReport), ctypes.sizeof(_lib.BasisOpts), _lib.BasisOpts.num_samples.offset]
    assert got == want


def test_feature_tiles_layout():
    import numpy as np
    # the network kernel's input tiles: BF16 (round to nearest even), row r at byte 128 r of
    # its tile, 16-byte chunk c at chunk position c ^ (r % 8)
    from its_b200.api import feature_tiles
    rng = np.random.default_rng(5)
    X = rng.standard_normal((300, 64)).astype(np.float32)
    t = feature_tiles(X)
    assert t.size == 3 * 16384
    words = t.view(np.uint16)
    bits = X.view(np.uint32).astype(np.uint64)
    bf = ((bits + 0x7FFF + ((bits >> 16) & 1)) >> 16).astype(np.uint16)
    for r in (0, 5, 127, 128, 201, 299):
        for c in range(8):
            base = (r // 128) * 8192 + (r % 128) * 64 + ((c ^ (r % 8)) & 7) * 8
            assert np.array_equal(words[base:base + 8], bf[r, 8 * c:8 * c + 8])
    assert not words[(300 % 128) * 64 + 2 * 8192:].any()  # rows past n are zero
