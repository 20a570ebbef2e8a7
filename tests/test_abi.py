"""The C-ABI libraries load without a GPU and export every declared entry point."""
import ctypes as C
import os
import re

import pytest

import nbk

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    txt = open(os.path.join(ROOT, "include", header)).read()
    return sorted(set(re.findall(r"NBK_API\s+[\w\s\*]+?\b(nbk_\w+)\s*\(", txt)))


@pytest.mark.parametrize("header,lib", [("nbk.h", "libnbk.so"), ("nbk_host.h", "libnbk_host.so")])
def test_library_exports_every_declared_symbol(header, lib):
    names = _declared(header)
    assert len(names) >= 8
    L = C.CDLL(os.path.join(ROOT, "namd-3.0_b200", lib))
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_errors_are_returned_not_raised():
    L = nbk.dev_lib()
    # NULL arguments are rejected with a status code and a message
    assert L.nbk_create(0, None, None) == -1
    assert b"NULL" in L.nbk_last_error()
    assert L.nbk_update_computes(None, 0, None, None) == -1
    assert L.nbk_destroy(None) == 0


def test_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lj = (1, [1.0], [1.0], [1.0], [1.0])
    with pytest.raises(nbk.NbkError):
        nbk.Nonbonded(nbk.NonbondedParams(), lj)


def test_record_layouts_match_reference():
    """Array strides of the records the boundary shares with the reference.
    CUDA's int2 is 8-byte aligned, so CudaComputeRecord {int2, float3} is 24
    bytes and TileList 48 (src/CudaTileListKernel.h:10-22,47-50); a caller's
    arrays of the reference structs must pass through unchanged."""
    assert C.sizeof(nbk.ComputeRecord) == 24
    assert C.sizeof(nbk.TileList) == 48
    assert C.sizeof(nbk.PatchRecord) == 16
    assert C.sizeof(nbk.TileExcl) == 128
    assert C.sizeof(nbk.Exclusion) == 32
    assert C.sizeof(nbk.VirialEnergy) == 31 * 8
    assert nbk.ComputeRecord.offsetXYZ.offset == 8
    assert nbk.TileList.patchInd.offset == 24 and nbk.TileList.icompute.offset == 40


def test_header_compiles_as_c_with_reference_strides(tmp_path):
    """include/nbk.h is plain C: a C translation unit sees the same record
    sizes, including the 128-byte CudaLocalRecord of the GPU-resident calls."""
    import subprocess
    src = tmp_path / "abi.c"
    src.write_text(
        '#include "nbk.h"\n'
        "_Static_assert(sizeof(nbk_compute_record) == 24, \"compute record\");\n"
        "_Static_assert(sizeof(nbk_tile_list) == 48, \"tile list\");\n"
        "_Static_assert(sizeof(nbk_local_record) == 128, \"local record\");\n"
        "_Static_assert(sizeof(nbk_pme_grid) == 16, \"pme grid\");\n"
        "_Static_assert(sizeof(nbk_double3) == 24, \"double3\");\n"
        "int main(void) { return 0; }\n")
    r = subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                        "-c", str(src), "-o", str(tmp_path / "abi.o")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_pme_and_resident_entry_points_reject_bad_arguments():
    L = nbk.dev_lib()
    vp = C.c_void_p
    assert L.nbk_pme_create(0, None, 0.3, None) == -1
    g = nbk.PmeGrid(4, 4, 4, 4)                 # grid below the minimum size
    h = vp()
    assert L.nbk_pme_create(0, C.byref(g), 0.3, C.byref(h)) == -1
    g = nbk.PmeGrid(32, 32, 32, 5)              # unsupported order
    assert L.nbk_pme_create(0, C.byref(g), 0.3, C.byref(h)) == -1
    assert L.nbk_pme_spread_charge(None, 0, None, None) == -1
    assert L.nbk_pme_destroy(None) == 0
    assert L.nbk_sort_patch_atoms(1, None, 64, None, None, None, None, None, None, None) == -1
    assert L.nbk_set_compute_positions(1, None, None, None, None, 1.0, None, None, None, None,
                                       None, None) == -1
    assert L.nbk_update_vdw_types_excl_device(None, 1, 32, None, None, None, None, None, None) == -1
    assert L.nbk_accumulate_forces_to_soa(None, 2, 1, *([None] * 5), 0, None,
                                          *([None] * 9), None) == -1
