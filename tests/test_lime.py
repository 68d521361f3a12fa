"""SciDAC LIME reader/writer (jaxqft_b200.lime) against the reference's own
reader: the golden LIME files were decoded by jaxqft/io/lime.py
(decode_scidac_gauge / decode_scidac_pseudofermion) into golden_lime.npz.
Host logic only (torch CPU device here; the GPU path only changes the device
of the final permute)."""

import os
import shutil

import numpy as np
import pytest
import torch

from jaxqft_b200 import lime
from tests.conftest import GOLDEN, load_golden


def test_gauge_files_decode_like_the_reference():
    g = load_golden("lime")
    for p in ("D", "F"):
        U = lime.load_gauge(os.path.join(GOLDEN, f"gauge_{p}.lime"), device="cpu").numpy()
        assert U.shape == g[f"U_{p}"].shape
        assert np.array_equal(U, g[f"U_{p}"]), p
    assert np.array_equal(g["U_D"][0], g["U"])  # the D file is exact
    assert np.abs(g["U_F"][0] - g["U"]).max() < 1e-6
    U2 = lime.load_gauge(os.path.join(GOLDEN, "gauge_D.lime"), batch_size=2, device="cpu")
    assert U2.shape[0] == 2 and torch.equal(U2[0], U2[1])


def test_fermion_and_momentum_decode():
    g = load_golden("lime")
    psi, fd = lime.load_fermion(os.path.join(GOLDEN, "fermion_D.lime"), device="cpu")
    assert fd.spins == 4 and fd.colors == 3
    assert np.array_equal(psi.numpy(), g["psi"])
    P, info = lime.load_momentum(os.path.join(GOLDEN, "gauge_D.lime"), device="cpu")
    assert info["rel_antihermitian_error"] > 0.1  # links are not algebra elements


def test_records_and_metadata():
    recs = list(lime.records(os.path.join(GOLDEN, "gauge_D.lime")))
    assert [r.type for r in recs] == ["scidac-private-file-xml", "scidac-private-record-xml", "scidac-binary-data"]
    assert recs[-1].nbytes == 2 * 4 * 4 * 6 * 4 * 9 * 16
    (fd,) = lime.fields(os.path.join(GOLDEN, "gauge_D.lime"))
    assert fd.dims == (2, 4, 4, 6) and fd.datacount == 4 and fd.precision == "D" and fd.colors == 3


def test_round_trip_and_errors(tmp_path):
    rng = np.random.default_rng(2)
    U = rng.standard_normal((4, 2, 2, 4, 2, 3, 3)) + 1j * rng.standard_normal((4, 2, 2, 4, 2, 3, 3))
    fn = tmp_path / "u.lime"
    lime.save_gauge(fn, U)
    assert np.array_equal(lime.load_gauge(fn, device="cpu").numpy()[0], U)
    bad = tmp_path / "bad.lime"
    data = bytearray(open(fn, "rb").read())
    data[0] ^= 0xFF
    bad.write_bytes(bytes(data))
    with pytest.raises(ValueError, match="not a LIME record"):
        lime.load_gauge(bad, device="cpu")
    short = tmp_path / "short.lime"
    short.write_bytes(open(fn, "rb").read()[:-100])
    with pytest.raises(ValueError):
        lime.load_gauge(short, device="cpu")
    psi_file = tmp_path / "f.lime"
    shutil.copy(os.path.join(GOLDEN, "fermion_D.lime"), psi_file)
    with pytest.raises(ValueError, match="ColorMatrix"):
        lime.load_gauge(psi_file, device="cpu")
