"""C-ABI surface checks that need no GPU: exported symbols, struct layouts, host helpers."""
from __future__ import annotations

import ctypes as C
import re
import subprocess
import textwrap

import numpy as np
import pytest

from conftest import ROOT

HEADER = ROOT / "include" / "icp_b200.h"


def declared_functions() -> list[str]:
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:[A-Za-z_][\w ]*?[\s\*]+)(icp_\w+)\s*\(", text, flags=re.M)))


def test_every_declared_function_is_exported(icp):
    names = declared_functions()
    assert "icp_hex_trace_bin" in names and "icp_phase_cdf_build" in names
    lib = C.CDLL(str(icp.LIB_PATH))
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) <= set(icp.exported_symbols()) | set(names)


def test_struct_layouts_match_c(icp, tmp_path):
    structs = {"icp_grid": icp.Grid, "icp_trace_stats": icp.TraceStats, "icp_tuning": icp.Tuning,
               "icp_hex_node": icp.HexNode, "icp_cdf_policy": icp.CdfPolicy, "icp_cdf_report": icp.CdfReport,
               "icp_hex_record": icp.HexRecordArgs, "icp_orientation": icp.Orientation,
               "icp_record_report": icp.RecordReport, "icp_drop_record": icp.DropRecordArgs,
               "icp_drop_report": icp.DropReport, "icp_drop_item": icp.DropItem,
               "icp_batch_settings": icp.BatchSettings, "icp_surrogate_config": icp.SurrogateConfig,
               "icp_adam": icp.Adam}
    src = tmp_path / "sizes.c"
    src.write_text('#include "icp_b200.h"\n#include <stdio.h>\nint main(void){\n' +
                   "".join(f'printf("{k} %zu\\n", sizeof({k}));\n' for k in structs) + "return 0;}\n")
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True).stdout.splitlines())
    for name, cls in structs.items():
        assert int(out[name]) == C.sizeof(cls), name


def test_u_edges_bit_identical_to_oracle(icp, oracle):
    for n in (1, 2, 3, 36, 72, 512, 900, 1801):
        assert np.array_equal(icp.u_edges(n), oracle.u_edges(n))


def test_frames_and_rotations_match_oracle(icp, oracle):
    rng = np.random.default_rng(2)
    for _ in range(50):
        k = rng.normal(size=3)
        ok, oe0, oe1 = oracle.make_frame(k)
        pk, pe0, pe1 = icp.make_frame(k)
        assert list(ok) == pk and list(oe0) == pe0 and list(oe1) == pe1
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        q = [float(x) for x in q]
        try:
            rot = oracle.rotation_from_quaternion(q)
        except ValueError:
            continue
        mine = np.array(icp.rotation_from_quaternion(*q)).reshape(3, 3).T
        assert np.array_equal(rot, mine)


def test_node_area_matches_oracle(icp, oracle):
    grid = icp.make_phase_grid(8, 16, (1, -0.4, 0.3))
    for q in [(1, 0, 0, 0), (0.5, 0.5, 0.5, 0.5)]:
        n = icp.HexNode()
        n.circumradius_mm, n.length_mm = 0.07, 0.3
        for i, v in enumerate(icp.rotation_from_quaternion(*q)):
            n.rotation[i] = v
        area = C.c_double()
        icp.check(icp.LIB.icp_hex_node_area(C.byref(n), C.byref(grid.abi()), C.byref(area)))
        rot = np.array(icp.rotation_from_quaternion(*q))
        expect = oracle.lib().icpo_hex_node_area(0.07, 0.3, rot.ctypes.data_as(oracle._D),
                                                 np.array(grid.ki).ctypes.data_as(oracle._D))
        assert area.value == expect


def test_orientation_plan_contract(icp):
    # hex_phase/tests/phase_tests.cpp:28-42
    header = "qw,qx,qy,qz,weight,samples,seed\n"
    p = icp.parse_orientation_plan("# explicit\r\n" + header + "1,0,0,0,0.25,17,18446744073709551615\r\n1,0,0,0,0.75,55,3\n")
    assert p.total_samples == 72 and len(p.nodes) == 2 and p.nodes[1].weight == 0.75
    for bad in ["1,0,0,0,2,1,1\n", "2,0,0,0,1,1,1\n", "1,0,0,0,nan,1,1\n", "1,0,0,0,1,0,1\n", "1,0,0,0,1,1,1,2\n",
                "1,0,0,0,0.5,18446744073709551615,1\n1,0,0,0,0.5,1,2\n"]:
        with pytest.raises(ValueError):
            icp.parse_orientation_plan(header + bad)
    assert icp.parse_orientation_plan(header + "1,0,0,0,1,5,1\n").source_sha256 == \
        __import__("hashlib").sha256((header + "1,0,0,0,1,5,1\n").encode()).hexdigest()


def test_context_fails_loudly_without_device(icp):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(icp.IcpError):
        icp.Context(0)
