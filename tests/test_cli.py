"""The ccmpred-compatible command line (ccmpred_b200/ccmpred).  CPU tests cover
argument and input errors (no GPU touched); GPU tests run the whole pipeline
and compare the .mat with the reference's post-processing of the written raw
couplings, byte for byte."""
import os
import subprocess

import numpy as np
import pytest

from ccmpred_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "ccmpred_b200", "ccmpred")
LETTERS = "ARNDCQEGHILKMFPSTWYV-"   # state -> letter (src/sequence.c:14-18)


def write_aln(path, msa):
    with open(path, "w") as f:
        for row in msa:
            f.write("".join(LETTERS[v] for v in row) + "\n")


def run(args, **kw):
    return subprocess.run([CLI] + args, capture_output=True, text=True, timeout=600, **kw)


def test_cli_usage_and_input_errors(tmp_path):
    assert os.path.exists(CLI)
    r = run([])
    assert r.returncode == 1 and "Usage" in r.stdout
    r = run([str(tmp_path / "missing.aln"), str(tmp_path / "o.mat")])
    assert r.returncode == 2 and "Cannot open" in r.stdout
    p = tmp_path / "x.fasta"
    p.write_text(">s1\nACDEF\n")
    r = run([str(p), str(tmp_path / "o.mat")])
    assert r.returncode == 100 and "PSICOV" in r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("flags", [[], ["-A"], ["-R"], ["-w", "0.7", "-l", "0.3"]])
def test_cli_end_to_end(gpu, ref_mod, tmp_path, flags):
    msa = synth.generate(synth.MSAConfig("cli", 30, 400, n_pairs=5, dup_frac=0.2, seed=71))
    aln = tmp_path / "in.aln"
    write_aln(aln, msa)
    mat, raw = tmp_path / "out.mat", tmp_path / "out.raw"
    r = run(["-n", "25", "-r", str(raw)] + flags + [str(aln), str(mat)])
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Output can be found in" in r.stdout
    lines = mat.read_text().splitlines()
    assert len(lines) == 30 and all(len(l.split("\t")) == 31 for l in lines)  # trailing tab
    # the .mat is the reference's sum_submatrices (+apc, +normalize) of the couplings
    x = ref_mod.ref_read_raw(str(raw), 30)
    cmap = ref_mod.ref_contact_map(x, 30, apc="-A" not in flags, normalize="-R" in flags)
    ref_mod.ref_write_matrix(str(tmp_path / "ref.mat"), cmap)
    assert mat.read_bytes() == (tmp_path / "ref.mat").read_bytes()
    # progress lines: iteration numbers 1..n
    it = [int(l.split("\t")[0]) for l in r.stdout.splitlines()
          if l[:1].isdigit() and len(l.split("\t")) == 6]
    assert it[:3] == [1, 2, 3]


@pytest.mark.gpu
def test_cli_warm_start_roundtrip(gpu, tmp_path):
    msa = synth.generate(synth.MSAConfig("cli2", 20, 300, n_pairs=3, seed=72))
    aln = tmp_path / "in.aln"
    write_aln(aln, msa)
    r1 = run(["-n", "10", "-r", str(tmp_path / "a.raw"), str(aln), str(tmp_path / "a.mat")])
    assert r1.returncode == 0, r1.stdout
    r2 = run(["-n", "10", "-i", str(tmp_path / "a.raw"), "-r", str(tmp_path / "b.raw"),
              str(aln), str(tmp_path / "b.mat")])
    assert r2.returncode == 0, r2.stdout
    f1 = float(r1.stdout.split("Final fx = ")[1].split()[0])
    f2 = float(r2.stdout.split("Final fx = ")[1].split()[0])
    assert f2 < f1
