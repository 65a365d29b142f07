"""Shared test set-up: the gpu marker, import paths, and the oracle's case dumps.

Cases are produced by the oracle (oracle/_ref/spo_ref_tool, the reference compiled from its own
sources) from the inputs in tests/golden: the boundary data of a run (the case bundle) plus the
reference CPU path's results for it. They are made once per session in a temporary directory.
"""

import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("", "cpp-spo-dvr_b200", "oracle"):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")
REF_TOOL = os.path.join(ROOT, "oracle", "_ref", "spo_ref_tool")
REF_FFT_CHECK = os.path.join(ROOT, "oracle", "_ref", "ref_fft_check")
TINY_CASES = ["tiny_hardwall", "tiny_dailight", "tiny_dailight_hetero", "tiny_oblique", "tiny_dailight_sym",
              "tiny_dailight_hetero_sym"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _ensure_built():
    """Builds the oracle and the product library when they are missing and their sources exist."""
    reference = os.environ.get("SPODVR_REFERENCE")
    if not os.path.exists(REF_TOOL):
        if not reference or not os.path.isdir(reference):
            pytest.fail(f"the oracle {REF_TOOL} is not built: run __graft_entry__.build(), or set SPODVR_REFERENCE "
                        "to the reference checkout and run make -C oracle")
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "-j8", "all", f"SPODVR_REFERENCE={reference}"],
                       check=True, stdout=subprocess.DEVNULL)
    lib = os.path.join(ROOT, "cpp-spo-dvr_b200", "lib", "libspo_b200.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-C", os.path.join(ROOT, "cpp-spo-dvr_b200"), "-j4"], check=True, stdout=subprocess.DEVNULL)


@pytest.fixture(scope="session")
def ref_case(tmp_path_factory):
    """ref_case(name, seed=7, analysis_steps=2, stages=True, input_path=None) -> output directory of
    `spo_ref_tool case`: case/ (the bundle), psi_initial, chi_start, stage_*, chi_steps, bk_steps,
    psi_final, block_densities (see oracle/ref_tool.cpp)."""
    _ensure_built()
    if not os.path.exists(REF_TOOL):
        pytest.fail(f"the oracle {REF_TOOL} is not built (make -C oracle)")
    cache = {}
    base = tmp_path_factory.mktemp("ref_cases")

    def make(name, seed=7, analysis_steps=2, stages=True, input_path=None, no_psi=False):
        key = (name, seed, analysis_steps, stages, input_path, no_psi)
        if key in cache:
            return cache[key]
        out = os.path.join(str(base), f"{name}_{seed}_{analysis_steps}_{int(stages)}_{int(no_psi)}")
        path = input_path or os.path.join(GOLDEN, "inputs", name + ".json")
        cmd = [REF_TOOL, "case", path, out, "--analysis-steps", str(analysis_steps)]
        if seed is not None:
            cmd += ["--random", str(seed)]
        if stages:
            cmd.append("--stages")
        if no_psi:
            cmd.append("--no-psi")
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            pytest.fail(f"spo_ref_tool failed for {name}: {r.stderr}")
        cache[key] = out
        return out

    return make


def read_c128(path, shape=None):
    import numpy as np
    a = np.fromfile(path, dtype=np.complex128)
    return a.reshape(shape) if shape is not None else a


def rel_err(a, b):
    """max |a - b| / max |b| (the reference's relative_difference, tests/comparison.hpp)."""
    import numpy as np
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def rel_l2(a, b):
    import numpy as np
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))
