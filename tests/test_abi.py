"""CPU tests of the C ABI boundary: the library loads, exports every function include/ae_mpm.h
declares, the ctypes mirrors have the header's exact struct layouts, and without a GPU the
library fails loudly instead of computing on the CPU.  No compute call is made here."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

import ae_mpm as M

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ae_mpm.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = set(re.findall(r"\b(ae_mpm_[a-z0-9_]+)\s*\(", src))
    return sorted(names)


def exported_symbols(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], stdout=subprocess.PIPE, text=True, check=True).stdout
    return {ln.split()[-1] for ln in out.splitlines() if " T " in ln}


def test_library_exports_every_declared_function():
    lib = M.LIB_PATH
    assert os.path.exists(lib), "build() has not produced libae_mpm.so"
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if n not in exported_symbols(lib)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    assert sorted(M.SIGNATURES) == declared_functions()


def test_library_loads_and_binds():
    lib = M.load()
    assert lib.ae_mpm_abi_version() == 1
    o = M.exec_opts()
    assert o.precision == 32 and o.sort_interval == 1 and o.use_graph == 1 and o.svd_fp64_fallback == 1


LAYOUT_PROBE = r"""
#include <stdio.h>
#include <stddef.h>
#include "ae_mpm.h"
#define S(T) printf(#T " %zu\n", sizeof(T));
#define O(T, f) printf(#T "." #f " %zu\n", offsetof(T, f));
int main(void) {
  S(ae_mpm_material) O(ae_mpm_material, model) O(ae_mpm_material, bulk_modulus)
  S(ae_mpm_config) O(ae_mpm_config, grid_size) O(ae_mpm_config, substeps) O(ae_mpm_config, gravity)
  O(ae_mpm_config, damping) O(ae_mpm_config, use_sparse_grid)
  S(ae_mpm_grid) O(ae_mpm_grid, dx) O(ae_mpm_grid, origin)
  S(ae_mpm_particles) O(ae_mpm_particles, material_idx)
  S(ae_mpm_scene_desc) O(ae_mpm_scene_desc, dt) O(ae_mpm_scene_desc, materials) O(ae_mpm_scene_desc, max_particles)
  S(ae_mpm_exec_opts) O(ae_mpm_exec_opts, svd_fp64_fallback)
  S(ae_mpm_tune_result) S(ae_mpm_server_opts) O(ae_mpm_server_opts, exec)
  S(ae_mpm_request_result) O(ae_mpm_request_result, done_s)
  return 0;
}
"""

CTYPES = {"ae_mpm_material": M.Material, "ae_mpm_config": M.Config, "ae_mpm_grid": M.Grid,
          "ae_mpm_particles": M.ParticlesView, "ae_mpm_scene_desc": M.SceneDesc, "ae_mpm_exec_opts": M.ExecOpts,
          "ae_mpm_tune_result": M.TuneResult, "ae_mpm_server_opts": M.ServerOpts,
          "ae_mpm_request_result": M.RequestResult}


def test_ctypes_struct_layouts_match_the_header():
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "probe.c")
        exe = os.path.join(d, "probe")
        open(src, "w").write(LAYOUT_PROBE)
        subprocess.run(["gcc", "-O0", "-I" + os.path.join(ROOT, "include"), src, "-o", exe], check=True)
        out = subprocess.run([exe], stdout=subprocess.PIPE, text=True, check=True).stdout
    for line in out.splitlines():
        key, val = line.split()
        val = int(val)
        if "." in key:
            t, f = key.split(".")
            assert getattr(CTYPES[t], f).offset == val, key
        else:
            assert C.sizeof(CTYPES[key]) == val, key


def _have_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_have_gpu(), reason="checks the no-GPU failure path")
def test_no_gpu_fails_loudly_instead_of_falling_back():
    with pytest.raises(M.MpmError) as e:
        M.Context(0)
    assert e.value.code in (M.ECUDA, M.EINVAL)


def test_oracle_is_not_linked_by_the_product():
    # the product library must not depend on the CPU oracle
    out = subprocess.run(["ldd", M.LIB_PATH], stdout=subprocess.PIPE, text=True).stdout
    assert "oracle" not in out
    for root, _, files in os.walk(os.path.join(ROOT, "ae-engine_b200")):
        for f in files:
            # build_native.py compiles the oracle alongside the library; nothing else may touch it
            if f.endswith((".py", ".cu", ".cuh", ".hpp", ".cpp")) and f != "build_native.py":
                txt = open(os.path.join(root, f), encoding="utf-8").read()
                assert "import oracle" not in txt and "mpm_oracle" not in txt, f
