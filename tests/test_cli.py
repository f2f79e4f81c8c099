"""The cudaamica-compatible command line (cudamica_b200/cudaamica).

CPU: the params-file reading follows the reference's rules, quirks included
(src/params.c, src/config.c:12-213) -- checked through the configuration echo,
which is printed before any GPU work.
GPU: a fit of the c0 case run through the CLI from raw float32 data writes the
reference's output files; they are compared with the reference's own outputs
for the same inputs (tests/golden/ref_c0.npz).
"""
import os
import re
import subprocess

import numpy as np
import pytest

from cudamica_b200 import build as B
from golden.cases import CASES, prepared, raw_data

CLI = os.path.join(os.path.dirname(B.LIB), "cudaamica")


@pytest.fixture(scope="module")
def cli():
    B.build()
    assert os.path.exists(CLI)
    return CLI


def run(cli, wd, params_text):
    with open(os.path.join(wd, "case.in"), "w") as f:
        f.write(params_text)
    return subprocess.run([cli, "-f", "case.in"], cwd=wd, capture_output=True, text=True, timeout=600)


def echo(out):
    vals = {}
    for line in out.splitlines():
        m = re.match(r"^(\w+) (\S+)$", line)
        if m:
            vals[m.group(1)] = m.group(2)
    return vals


def small_data(wd, n=4, T=64):
    np.zeros((T, n), dtype=np.float32).tofile(os.path.join(wd, "data.fdt"))


BASE = ["datafile data.fdt", "nchannels 4", "nsamples 64", "spherefile sphere.fdt"]


def test_defaults_and_update_rho_quirk(cli, tmp_path):
    small_data(tmp_path)
    r = run(cli, tmp_path, "\n".join(BASE + ["do_newton off"]) + "\n")
    v = echo(r.stdout)
    # missing update_rho: rho stays fixed and do_newton is forced on
    assert (v["update_rho"], v["do_newton"]) == ("0", "1")
    assert (v["maxiter"], v["nsdm"], v["nmmodels"], v["do_sphere"]) == ("200", "3", "1", "1")
    assert v["datafile"] == "data.fdt"


def test_comment_line_is_skipped(cli, tmp_path):
    small_data(tmp_path)
    r = run(cli, tmp_path, "# nsdm 5\n" + "\n".join(BASE + ["update_rho 1", "maxiter 7"]) + "\n")
    v = echo(r.stdout)
    assert (v["nsdm"], v["maxiter"], v["update_rho"]) == ("3", "7", "1")


def test_substring_match_consumes_a_later_key(cli, tmp_path):
    # "nsdm" is looked up before "spherefile": its scan hits the spherefile line
    # first (substring), cuts it at the first space, and spherefile is then
    # malformed -- the reference's behaviour
    small_data(tmp_path)
    text = "\n".join(["datafile data.fdt", "nchannels 4", "nsamples 64",
                      "spherefile out/nsdm_sphere.fdt", "nsdm 2"]) + "\n"
    r = run(cli, tmp_path, text)
    assert r.returncode == 256 - 3, (r.returncode, r.stderr)
    assert "sphere file" in r.stderr
    text_ok = "\n".join(["datafile data.fdt", "nchannels 4", "nsamples 64", "nsdm 2",
                         "spherefile out/nsdm_sphere.fdt"]) + "\n"
    v = echo(run(cli, tmp_path, text_ok).stdout)
    assert v["nsdm"] == "2"


def test_string_value_loses_its_last_character(cli, tmp_path):
    small_data(tmp_path)
    # no newline after the last line: "data.fdt" is read as "data.fd"
    text = "\n".join(["nchannels 4", "nsamples 64", "spherefile sphere.fdt", "datafile data.fdt"])
    r = run(cli, tmp_path, text)
    assert echo(r.stdout)["datafile"] == "data.fd"
    assert r.returncode == 256 - 5                       # no such file


def test_missing_required_key(cli, tmp_path):
    small_data(tmp_path)
    r = run(cli, tmp_path, "\n".join(BASE[1:]) + "\n")  # no datafile
    assert r.returncode != 0 and "data file" in r.stderr


def test_truncated_data_file_is_reported(cli, tmp_path):
    # fewer than nsamples x nchannels float32 values: an error before any GPU work
    np.zeros((63, 4), dtype=np.float32).tofile(os.path.join(tmp_path, "data.fdt"))
    r = run(cli, tmp_path, "\n".join(BASE) + "\n")
    assert r.returncode == 256 - 5, (r.returncode, r.stderr)    # AMICA_ERR_NOFILE
    assert "cannot read 64 x 4 float32 values" in r.stderr


def test_truncated_initial_state_file_is_reported(cli, tmp_path):
    # ainitfile shorter than one n x n block
    small_data(tmp_path)
    np.zeros(15, dtype=np.float32).tofile(os.path.join(tmp_path, "a0.fdt"))
    r = run(cli, tmp_path, "\n".join(BASE + ["ainitfile a0.fdt"]) + "\n")
    assert r.returncode == 256 - 5, (r.returncode, r.stderr)


@pytest.mark.gpu
def test_cli_fit_matches_reference_outputs(cli, tmp_path):
    case = CASES["c0"]
    ref = np.load(f"{pytest.golden_dir}/ref_c0.npz")
    p = prepared(case)
    raw_data(case).astype(np.float32).tofile(tmp_path / "data.fdt")
    p["A0"].astype(np.float32).tofile(tmp_path / "a0.fdt")
    p["c0"].astype(np.float32).tofile(tmp_path / "c0.fdt")
    os.makedirs(tmp_path / "out")
    lines = ["datafile data.fdt", f"nchannels {case.n}", f"nsamples {case.T}", "do_sphere 1",
             f"maxiter {case.maxiter}", f"nsdm {case.m}", f"nmmodels {case.M}",
             "spherefile out/sphere.fdt", "block_size 5000", "fix_init on", "do_newton on",
             f"newt_start_iter {case.newt_start_iter}", "rho_start_iter 1",
             "weightsfile out/W.fdt", "afile out/A.fdt", "cfile out/c.fdt", "llfile out/ll.fdt",
             "ltallfile out/ltall.fdt", "gmfile out/gm.fdt", "alphafile out/alpha.fdt",
             "mufile out/mu.fdt", "betafile out/beta.fdt", "rhofile out/rho.fdt", "update_rho 1",
             "precision fp32", "ainitfile a0.fdt", "cinitfile c0.fdt"]
    r = run(cli, tmp_path, "\n".join(lines) + "\n")
    assert r.returncode == 0, r.stderr
    it = [(int(a), float(b), float(c)) for a, b, c in
          re.findall(r"Iteration (\d+): lrate (\S+) LL (\S+)", r.stdout)]
    assert len(it) == case.maxiter
    ll = np.array([t[2] for t in it])
    lr = np.array([t[1] for t in it])
    np.testing.assert_array_equal(lr, ref["lrate"])
    # FP32 E-step vs the reference's FP64 build: within 1e-5 nats per sample for
    # the first iterations; the trajectories then drift apart by up to ~2e-5 by
    # iteration 100 (the mu denominator sum u |y|^(rho-2) is dominated by the few
    # samples with y near 0, where FP32 b = W (x - c) differs in its leading digits)
    assert np.max(np.abs(ll[:20] - ref["ll"][:20])) < 1e-5
    assert np.max(np.abs(ll - ref["ll"])) < 3e-5
    rd = lambda name, shape: np.fromfile(tmp_path / "out" / name, dtype=np.float64).reshape(shape)
    n, M, m = case.n, case.M, case.m
    assert np.max(np.abs(rd("ll.fdt", (-1,)) - ll)) == 0.0
    assert np.max(np.abs(rd("sphere.fdt", (n, n)) - ref["sphere"])) < 1e-10
    # after 100 chaotic iterations even the FP64 oracle's W is 1.4e-3 (relative to
    # its largest entry) from the reference's; the FP32 fit must land in that band
    for name, key, shape in (("W.fdt", "W", (M, n, n)), ("A.fdt", "A", (M, n, n))):
        got = rd(name, shape)
        assert np.max(np.abs(got - ref[key])) / np.max(np.abs(ref[key])) < 3e-3, name
    # the FP64 oracle's mixture parameters land 4e-3 (alpha, rho), 5.8e-3 (mu) and
    # 8.3e-3 (beta) from the reference's after the same 100 iterations
    for name, key in (("alpha.fdt", "alpha"), ("beta.fdt", "beta"), ("rho.fdt", "rho"),
                      ("mu.fdt", "mu")):
        got = rd(name, (M, m, n))
        assert np.max(np.abs(got - ref[key])) / np.max(np.abs(ref[key])) < 2.5e-2, name
    assert np.max(np.abs(rd("gm.fdt", (M,)) - ref["gm"])) < 1e-12
    assert np.max(np.abs(rd("c.fdt", (M, n)) - ref["c"])) / np.max(np.abs(ref["c"])) < 2.5e-2
    assert os.path.getsize(tmp_path / "out" / "ltall.fdt") == 8 * M * case.T
