"""The C interface checked by a C99 program (tests/c/abi_smoke.c), as the
reference checks its own header (tools/check_c_abi.sh): compiled with
`cc -std=c99 -Wall -Wextra -Werror` against include/knappnet.h, so any
prototype of a reference entry point that drifted from the reference's
netcapi.h fails the build, linked to libknappnet_b200.so and run: host-only
calls on CPU, net_pagerank against the reference's hand values on a GPU.
"""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import pytest

import knappnet_b200 as K

ROOT = Path(__file__).resolve().parent.parent
SRC = ROOT / "tests" / "c" / "abi_smoke.c"
FLAGS = ["-std=c99", "-Wall", "-Wextra", "-Werror"]


def compiler():
    cc = shutil.which("cc") or shutil.which("gcc")
    if cc is None:
        pytest.skip("no C compiler")
    return cc


@pytest.fixture(scope="module")
def smoke(tmp_path_factory):
    cc = compiler()
    if not K.LIB_PATH.exists():
        pytest.skip("libknappnet_b200.so is not built")
    out = tmp_path_factory.mktemp("abi") / "abi_smoke"
    lib_dir = str(K.LIB_PATH.parent)
    cmd = [cc, *FLAGS, "-I", str(ROOT / "include"), str(SRC), "-L", lib_dir,
           "-l:" + K.LIB_PATH.name, "-Wl,-rpath," + lib_dir, "-lm", "-o", str(out)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


def test_c_program_compiles_and_runs_host_calls(smoke):
    r = subprocess.run([str(smoke), "cpu"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "cpu checks: ok" in r.stdout


def test_prototype_drift_fails_to_compile(tmp_path):
    """A pointer type that disagrees with the header's declaration (one
    parameter added) must not compile under -Werror: the check has teeth."""
    cc = compiler()
    good = SRC.read_text()
    bad = good.replace("typedef int64_t (*graph_count_t)(const GraphHandle *);",
                       "typedef int64_t (*graph_count_t)(const GraphHandle *, int32_t);")
    assert bad != good
    for name, text, ok in (("good.c", good, True), ("drift.c", bad, False)):
        f = tmp_path / name
        f.write_text(text)
        r = subprocess.run([cc, *FLAGS, "-I", str(ROOT / "include"), "-c", str(f), "-o",
                            str(tmp_path / (name + ".o"))], capture_output=True, text=True)
        assert (r.returncode == 0) == ok, r.stderr


@pytest.mark.gpu
def test_c_program_pagerank_on_gpu(smoke):
    r = subprocess.run([str(smoke), "gpu"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "gpu checks: ok" in r.stdout
