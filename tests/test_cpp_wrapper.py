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
