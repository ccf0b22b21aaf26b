"""Byte layouts (src/renderer.rs:2253-2261) and the C-ABI surface of libirt.so."""
import ctypes as C
import os
import re

from instantradiositytest_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_gpu_layout_sizes_match_wgsl():
    # gpu_layout_sizes_match_wgsl: Vertex 64, Mesh 128, Object 208, Light 48,
    # Material 64, Frame 384; plus Node, Vpl and Reservoir of common.wgsl.
    assert L.VERTEX_DTYPE.itemsize == 64
    assert L.MESH_DTYPE.itemsize == 128
    assert L.OBJECT_DTYPE.itemsize == 208
    assert L.LIGHT_DTYPE.itemsize == 48
    assert L.MATERIAL_DTYPE.itemsize == 64
    assert C.sizeof(L.Frame) == 384
    assert L.NODE_DTYPE.itemsize == 48
    assert L.VPL_DTYPE.itemsize == 48
    assert L.RESERVOIR_DTYPE.itemsize == 32


def test_frame_field_offsets():
    # common.wgsl:3-8 field order: four mat4, then eight vec4s.
    names = ["camera", "size", "counts", "restir", "temporal", "sdf", "rr", "flags"]
    for i, n in enumerate(names):
        assert getattr(L.Frame, n).offset == 256 + 16 * i


def declared_functions():
    text = open(os.path.join(ROOT, "include", "irt.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(irt_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(L.LIB_PATH)
    declared = declared_functions()
    assert len(declared) > 30
    missing = [n for n in declared if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding covers exactly the declared surface
    assert sorted(L.exported_symbols()) == declared


def test_settings_defaults_validate():
    s = L.Settings()
    L.lib.irt_settings_default(C.byref(s))
    msg = C.create_string_buffer(128)
    assert L.lib.irt_settings_validate(C.byref(s), msg, 128) == L.IRT_OK
    assert (s.render_width, s.render_height, s.vpl_count, s.restir_max_history, s.svgf_iterations) == (
        1920, 1200, 100, 4, 4)


def test_invalid_budgets_and_nonfinite_settings_are_rejected():
    # src/settings.rs:111-131
    edits = [
        ("render_width", 0, "invalid render size"),
        ("vpl_count", 0, "invalid VPL budget"),
        ("temporal_max_history", 0, "invalid temporal settings"),
        ("restir_max_history", 0, "invalid ReSTIR history/SVGF iteration count"),
        ("restir_max_history", 33, "invalid ReSTIR history/SVGF iteration count"),
        ("svgf_iterations", 0, "invalid ReSTIR history/SVGF iteration count"),
        ("svgf_iterations", 6, "invalid ReSTIR history/SVGF iteration count"),
        ("sdf_hit_epsilon", float("inf"), "invalid SDF settings"),
        ("vpl_rr_max_survival", 1.0, "invalid roulette probabilities"),
        ("depth_threshold", float("nan"), "invalid rejection/frame budget"),
    ]
    for field, value, message in edits:
        s = L.Settings()
        L.lib.irt_settings_default(C.byref(s))
        setattr(s, field, value)
        msg = C.create_string_buffer(128)
        assert L.lib.irt_settings_validate(C.byref(s), msg, 128) == L.IRT_E_INVALID, field
        assert msg.value.decode() == message


def test_context_without_device_reports_nodevice():
    # On a CPU-only host the context refuses with IRT_E_NODEVICE instead of
    # falling back to anything.
    import torch

    if torch.cuda.is_available():
        return
    h = C.c_void_p()
    cfg = L.Config(0, 0)
    assert L.lib.irt_context_create(C.byref(cfg), C.byref(h)) == L.IRT_E_NODEVICE


def test_checked_build_exports_the_same_abi():
    """libirt_checked.so (kernels test every data-dependent index) is the same
    C-ABI as libirt.so, and each reports its flavour."""
    assert os.path.exists(L.CHECKED_LIB_PATH), "build it with make -C instantradiositytest_b200"
    checked = C.CDLL(L.CHECKED_LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(checked, n)]
    assert not missing, missing
    checked.irt_build_flavour.restype = C.c_char_p
    assert checked.irt_build_flavour() == b"checked"
    assert L.lib.irt_build_flavour() == (b"checked" if L.LIB_PATH == L.CHECKED_LIB_PATH else b"default")


def test_reference_arm_loads_no_cuda_code():
    """bench.py's reference arm times the oracle; its inputs come from the
    host-only library (libirt_host.so: generator, CPU producers, loader), so
    the process maps neither libirt.so nor the CUDA runtime."""
    import json
    import subprocess
    import sys

    assert os.path.exists(L.HOST_LIB_PATH), "build it with make -C instantradiositytest_b200"
    code = ("import sys, runpy\n"
            "sys.argv = ['bench.py', '--impl', 'reference', '--config', '0', '--steps', '1', '--warmup', '1',"
            " '--reference-seconds', '1']\n"
            "runpy.run_path('bench.py', run_name='__main__')\n"
            "maps = open('/proc/self/maps').read()\n"
            "print('MAPS', 'libirt.so' in maps, 'libirt_host.so' in maps, 'libcudart' in maps)\n")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads([x for x in r.stdout.splitlines() if x.startswith("{")][-1])
    assert line["impl"] == "reference" and line["value"] > 0
    assert r.stdout.strip().splitlines()[-1] == "MAPS False True False"


def test_committed_profiles_hold_the_bench_figures():
    """bench.py takes the march's DRAM bytes per launch (the line's
    roofline traffic) for each storage and field sampler, and its executed
    FP32 flops per pixel, from the committed ncu summaries under profiles/."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("bench_figures", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    for workload in ("1920x1200", "1920x1200_mixed", "1920x1200_field_linear"):
        traffic = bench.ncu_traffic("march", workload)
        assert traffic is not None and 3.13e8 <= traffic < 2e9, (workload, traffic)
    flops = bench.ncu_figure("march", "1920x1200", "executed_fp32_flops_per_pixel")
    assert flops is not None and 1000 < flops < 20190
