"""single_dev_expt_main argv handling (CPU only: every case here fails or
exits before the device is touched)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "culbm_b200", "bin", "single_dev_expt_main")


def run(*args):
    if not os.path.exists(CLI):
        pytest.fail(f"{CLI} not built (python -m culbm_b200.build)")
    return subprocess.run([CLI, *args], capture_output=True, text=True, timeout=60)


def test_help_lists_every_reference_flag():
    r = run("--help")
    assert r.returncode == 0
    for flag in ("--devId", "--dstep", "--nstep", "--invTau", "--blockDim", "--gridDim", "--domainDim",
                 "--streamPolicy", "--optPolicy", "--velSet", "--initStateFolder", "--dumpFolder", "--dumpRho",
                 "--dumpVx", "--dumpVy", "--dumpVz", "--useRingDDFBuf", "--innerLoop"):
        assert flag in r.stdout, flag


@pytest.mark.parametrize("args,code", [
    (["--bogus"], 109),                      # CLI11 ExtrasError
    (["--nstep", "abc"], 104),               # CLI11 ConversionError
    (["--blockDim", "[32,16]"], 114),        # CLI11 ArgumentMismatch
    (["--dstep"], 114),
])
def test_parse_errors_use_cli11_exit_codes(args, code):
    r = run(*args)
    assert r.returncode == code, (r.returncode, r.stderr)
    assert r.stderr


def test_ring_buffer_outside_inplace_dynamic_l2_is_rejected():
    r = run("--useRingDDFBuf", "--streamPolicy", "0", "--optPolicy", "3")
    assert r.returncode == 1
    assert "--useRingDDFBuf is unimplemented unless --streamPolicy 1 --optPolicy 3." in r.stderr


def test_plain_pull_grid_must_cover_domain():
    r = run("--blockDim", "[32,16,2]", "--gridDim", "[2,3,19]", "--domainDim", "[256,256,256]")
    assert r.returncode == 1
    assert "Dimension of domain doesn't match computation grid!" in r.stderr


@pytest.mark.parametrize("form", [["--domainDim", "[64,48,40]"], ["--domainDim=[64,48,40]"],
                                  ["--domainDim", "64,48,40"], ["--domainDim", "64", "48", "40"]])
def test_vector_syntaxes_accepted(form):
    # A mismatching grid makes the run stop at the geometry check, after parsing.
    r = run(*form, "--blockDim", "[8,8,8]", "--gridDim", "[1,1,1]")
    assert r.returncode == 1
    assert "Dimension of domain doesn't match computation grid!" in r.stderr


@pytest.mark.parametrize("flag", ["--persistL2", "--noPersistL2", "--noCacheHints", "--noGraphs"])
def test_addition_flags_parse(flag):
    # Accepted flags reach the geometry check, which stops the run before the device.
    r = run(flag, "--domainDim", "[64,48,40]", "--blockDim", "[8,8,8]", "--gridDim", "[1,1,1]")
    assert r.returncode == 1, (r.returncode, r.stderr)
    assert "Dimension of domain doesn't match computation grid!" in r.stderr
    assert "--persistL2" in run("--help").stdout
