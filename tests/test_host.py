"""Host-side drop-in pieces vs the compiled reference, bit-for-bit (CPU)."""
import os

import numpy as np
import pytest

from ccmpred_b200 import host, synth


@pytest.mark.parametrize("L,N,seed", [(9, 31, 1), (40, 300, 2), (75, 1000, 3)])
def test_init_bias_bit_exact(ref_mod, L, N, seed):
    msa = synth.generate(synth.MSAConfig("t", L, N, seed=seed))
    a = host.init_bias(msa)
    b = ref_mod.ref_init_bias(msa)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("apc,norm", [(True, False), (False, False), (True, True)])
def test_contact_map_bit_exact(ref_mod, apc, norm):
    L = 17
    x = synth.random_x(L, 4, w_sd=0.1)
    a, xnorm = host.contact_map(x, L, apc=apc, normalize=norm)
    b = ref_mod.ref_contact_map(x, L, apc=apc, normalize=norm)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert xnorm > 0


def test_contact_map_golden(oracle_mod):
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "eval_L9_N31_rand.npz"))
    a, _ = host.contact_map(d["x"], 9, apc=True)
    assert np.array_equal(a.view(np.uint32), d["contact_map_apc"].view(np.uint32))


def test_output_files_byte_identical(ref_mod, tmp_path):
    L = 11
    x = synth.random_x(L, 6, w_sd=0.1)
    mat, _ = host.contact_map(x, L)
    host.write_matrix(str(tmp_path / "a.mat"), mat)
    ref_mod.ref_write_matrix(str(tmp_path / "b.mat"), mat)
    assert (tmp_path / "a.mat").read_bytes() == (tmp_path / "b.mat").read_bytes()
    host.write_raw(str(tmp_path / "a.raw"), x, L)
    ref_mod.ref_write_raw(str(tmp_path / "b.raw"), x, L)
    assert (tmp_path / "a.raw").read_bytes() == (tmp_path / "b.raw").read_bytes()
    xa = host.read_raw(str(tmp_path / "a.raw"), L)
    xb = ref_mod.ref_read_raw(str(tmp_path / "b.raw"), L)
    assert np.array_equal(xa.view(np.uint32), xb.view(np.uint32))


def test_read_msa_matches_reference(ref_mod, tmp_path):
    path = ref_mod.REF_EXAMPLE_ALN
    if not os.path.exists(path):
        pytest.skip("reference example alignment not copied into oracle/_ref")
    a = host.read_msa(path)
    b = ref_mod.ref_read_msa(path)
    assert a.shape == (3068, 75) and np.array_equal(a, b)
    p = tmp_path / "x.fasta"
    p.write_text(">seq\nACDE\n")
    with pytest.raises(ValueError):
        host.read_msa(str(p))


def test_read_msa_alphabet(tmp_path):
    p = tmp_path / "t.aln"
    p.write_text("ARNDCQEGHILKMFPSTWYV-\nBJOUXZ.acd-\n")
    m = host.read_msa(str(p))
    assert m.shape == (2, 21)
    assert list(m[0]) == list(range(21))
    assert list(m[1][:6]) == [20] * 6 and list(m[1][7:10]) == [0, 4, 3]
