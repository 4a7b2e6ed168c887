"""The C ABI library loads and exports every function include/sbh_b200.h declares,
and the pybind11 modules expose the reference plugin's names.  No GPU needed."""
import ctypes
import os
import re

import sbh
import sbh_capi as C
import sbh_gpu
from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "sbh_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sbh_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(C.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert missing == []


def test_ctypes_binding_covers_the_header():
    assert sorted(C._SIGNATURES) == declared_functions()


STRUCTS = {  # C name -> ctypes mirror
    "sbh_params": C.Params, "sbh_tree_info": C.TreeInfo, "sbh_batch_item": C.BatchItem,
    "sbh_batch_tuning": C.BatchTuning, "sbh_server_config": C.ServerConfig,
    "sbh_request_info": C.RequestInfo, "sbh_server_stats": C.ServerStats,
}


def test_struct_layouts_match_the_c_compiler(tmp_path):
    """Size and every field offset of each ABI struct, as gcc lays it out from
    the header, equal the ctypes mirror's."""
    import shutil
    import subprocess

    import pytest
    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    lines = ["#include <stddef.h>", "#include <stdio.h>", f'#include "{HEADER}"',
             "int main(void) {"]
    for cname, cls in STRUCTS.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in cls._fields_:
            lines.append(f'  printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-o", str(exe), str(src)], check=True)
    got = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True,
                               text=True).stdout.splitlines():
        cname, what, v = line.split()
        got[(cname, what)] = int(v)
    for cname, cls in STRUCTS.items():
        assert got[(cname, "size")] == ctypes.sizeof(cls), cname
        for field, _ in cls._fields_:
            assert got[(cname, field)] == getattr(cls, field).offset, (cname, field)
    assert C.lib().sbh_abi_version() == 1


def test_status_strings():
    assert C.lib().sbh_status_string(0) == b"ok"
    assert C.lib().sbh_status_string(5) == b"device-side iteration limit hit"


def test_reference_plugin_surface():
    for cls in ("QuadtreeGPU1", "QuadtreeGPU2", "QuadtreeGPU3", "OctreeGPU1", "OctreeGPU2",
                "OctreeGPU3"):
        assert hasattr(sbh_gpu, cls)
    for k in ("gravity", "wn", "smoothdist"):
        for f in ("eval_brute_force_", "eval_barnes_hut_", "multi_level_prefix_control_variate_"):
            assert hasattr(sbh_gpu, f + k)
        assert hasattr(sbh, "eval_barnes_hut_" + k)
        assert hasattr(sbh, "multi_level_prefix_control_variate_" + k)
    for cls in ("Quadtree1", "Quadtree2", "Quadtree3", "Octree1", "Octree2", "Octree3"):
        assert hasattr(sbh, cls)


def test_batch_tuning_defaults_and_range_checks():
    """sbh_batch_tuning_init's defaults, and sbh_batch_set_tuning's refusals,
    which happen on the host before any device is touched."""
    t = C.batch_tuning()
    assert t.as_dict() == {"sampler_unit_queries": 32, "bucket_queries": 8, "blocks_per_sm": 0,
                           "bh_unit_queries": 32, "direct_queries": 65536}
    import pytest
    for bad in (dict(sampler_unit_queries=0), dict(bucket_queries=1), dict(blocks_per_sm=-1),
                dict(bh_unit_queries=33), dict(direct_queries=-1)):
        with pytest.raises(C.SbhError):
            C.set_batch_tuning(C.batch_tuning(**bad))
