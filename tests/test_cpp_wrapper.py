"""The header-only C++ API (include/gmapf/GMAPF.h) compiled into a
reference-style client and run: lifecycle rules on the CPU, and a full run
on the GPU checked against the oracle world."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from gmapf_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "cpp" / "wrapper_demo.cpp"


@pytest.fixture(scope="module")
def demo(tmp_path_factory):
    _lib.load()
    exe = tmp_path_factory.mktemp("cpp") / "wrapper_demo"
    libdir = _lib.LIB_PATH.parent
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", str(ROOT / "include"), str(SRC), "-o", str(exe),
                    "-L", str(libdir), "-lgmapf_b200", f"-Wl,-rpath,{libdir}"], check=True)
    return exe


def test_cpp_wrapper_lifecycle(demo):
    r = subprocess.run([str(demo), "cpu"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "cpu ok thrown=2" in r.stdout
    assert "state=1" in r.stdout  # Search after SetAgentTargetPos (GMAPF.cu:248)


@pytest.mark.gpu
def test_cpp_wrapper_run_matches_oracle(demo, oracle_mod):
    import gmapf_b200 as G
    from gmapf_b200 import scenarios as S
    r = subprocess.run([str(demo), "gpu"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    rows = [ln.split() for ln in r.stdout.splitlines() if ln.startswith("agent ")]
    got_pos = np.array([[float(a[2]), float(a[3])] for a in rows], np.float32)
    got_state = np.array([int(a[4]) for a in rows])
    assert "[gmapf] step avg:" in r.stdout

    scn = S.zigzag()
    g = G.GMAPF()
    g.Init(G.make_config(4, 2, 1, 4, 4, 16))
    S.build_map(g, scn)
    om = oracle_mod.OMap(g.map_nodes())
    A = 256
    ow = oracle_mod.OWorld(om, A, 2.0, 1.0, A, 4, 16, 1.0)
    for i in range(A):
        assert ow.add_agent(i / 5.0 + 1.0, 1.0) == i
    for i in range(A):
        assert ow.set_target(i, i / 5.0 + 1.0, 950.0) == 0
    for _ in range(120):
        ow.step(np.float32(1.0 / 60.0), 8)
    o = ow.get()
    assert np.array_equal(got_state, o["state"])
    assert np.allclose(got_pos, o["pos"], rtol=1e-4, atol=1e-4, equal_nan=True)


@pytest.mark.gpu
def test_cpp_scene_batch_matches_oracle(demo, oracle_mod):
    import gmapf_b200 as G
    from gmapf_b200 import scenarios as S
    r = subprocess.run([str(demo), "batch"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    rows = [ln.split() for ln in r.stdout.splitlines() if ln.startswith("scene ")]
    assert "served completed=16 found=16 applied=16" in r.stdout
    g = G.GMAPF()
    g.Init(G.make_config(4, 2, 1, 4, 4, 16))
    S.build_map(g, S.zigzag())
    om = oracle_mod.OMap(g.map_nodes())
    A = 128
    f32 = np.float32
    for k, radius in enumerate([2.0, 1.5]):
        ow = oracle_mod.OWorld(om, A, radius, 1.0, A, 4, 16, 1.0)
        for i in range(A):  # the demo's float arithmetic
            x0 = f32(i) / f32(5) + f32(1) if k == 0 else f32(i) / f32(4) + f32(2)
            assert ow.add_agent(x0, f32(1) if k == 0 else f32(3)) == i
        for i in range(A):
            x1 = f32(i) / f32(5) + f32(1) if k == 0 else f32(990) - f32(i) / f32(4)
            assert ow.set_target(i, x1, f32(950) if k == 0 else f32(600)) == 0
        for _ in range(120):
            ow.step(np.float32(1.0 / 60.0), 8)
        o = ow.get()
        mine = [a for a in rows if a[1] == str(k)]
        pos = np.array([[float(a[4]), float(a[5])] for a in mine], np.float32)
        st = np.array([int(a[6]) for a in mine])
        assert np.array_equal(st, o["state"]), f"scene {k} states"
        assert np.allclose(pos, o["pos"], rtol=1e-4, atol=1e-4, equal_nan=True), f"scene {k} positions"
