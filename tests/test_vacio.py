"""VAC configuration files (the reference's ascii .ini and binary .out
formats): round trips, the byte layout of the binary format, and the
reference's own configuration files where its sources are present."""
from __future__ import annotations

import struct
from pathlib import Path

import numpy as np
import pytest

from smaug_b200 import SmaugError, problems
from smaug_b200 import vacio

from oracle.ref_shim import reference_root

_REF = reference_root()
REF_CONFIGS = _REF / "dev" / "smaug" / "configs" if _REF else Path("/nonexistent")


def test_ascii_round_trip_is_exact(tmp_path):
    prob = problems.orszag_tang(20, ny=12, rho_noise=0.01, seed=3)
    pos = vacio.positions(prob)
    hdr = vacio.header_for(prob, it=7, t=0.125)
    vacio.write_ascii(tmp_path / "ot.ini", hdr, pos, prob.w)
    h, p2, w2 = vacio.read_ascii(tmp_path / "ot.ini")
    assert (h["it"], h["t"], h["ndim"], h["nw"], h["n"]) == (7, 0.125, 2, 10, (24, 16))
    assert h["eqpar"][0] == prob.gamma
    assert np.array_equal(p2, pos) and np.array_equal(w2, prob.w)


def test_binary_round_trip_and_layout(tmp_path):
    prob = problems.blast_wave(6, seed=2)
    pos = vacio.positions(prob)
    hdr = vacio.header_for(prob, it=3, t=0.5)
    f = tmp_path / "bw_3.out"
    vacio.write_binary(f, hdr, pos, prob.w)
    h, p2, w2 = vacio.read_binary(f)
    assert (h["it"], h["t"], h["ndim"], h["nw"], h["n"]) == (3, 0.5, 3, 13, (10, 10, 10))
    assert np.array_equal(p2, pos) and np.array_equal(w2, prob.w)
    # the byte layout of writevacconfig (src/readwrite.c:160-368)
    raw = f.read_bytes()
    o = 79
    it, = struct.unpack_from("<i", raw, o)
    t, = struct.unpack_from("<d", raw, o + 4)
    ndim, neq, nw = struct.unpack_from("<3i", raw, o + 12)
    n = struct.unpack_from(f"<{ndim}i", raw, o + 24)
    o = o + 24 + 4 * ndim + 8 * neq + 79
    N = int(np.prod(n))
    body = np.frombuffer(raw, dtype="<f8", count=(ndim + nw) * N, offset=o)
    assert (it, t, ndim, nw, n) == (3, 0.5, 3, 13, (10, 10, 10))
    assert np.array_equal(body[:ndim * N].reshape(pos.shape), pos)
    assert np.array_equal(body[ndim * N:].reshape(prob.w.shape), prob.w)
    assert len(raw) == o + 8 * (ndim + nw) * N + 1 and raw[-1:] == b"\n"


def test_truncated_files_are_errors(tmp_path):
    prob = problems.orszag_tang(8)
    vacio.write_ascii(tmp_path / "a.ini", vacio.header_for(prob), vacio.positions(prob), prob.w)
    text = (tmp_path / "a.ini").read_text().splitlines()
    (tmp_path / "b.ini").write_text("\n".join(text[:-3]) + "\n")
    with pytest.raises(SmaugError):
        vacio.read_ascii(tmp_path / "b.ini")
    vacio.write_binary(tmp_path / "a.out", vacio.header_for(prob), vacio.positions(prob), prob.w)
    (tmp_path / "b.out").write_bytes((tmp_path / "a.out").read_bytes()[:-100])
    with pytest.raises(SmaugError):
        vacio.read_binary(tmp_path / "b.out")


def test_problem_from_vac_pads_inner_cells(tmp_path):
    prob = problems.orszag_tang(16)
    inner = (slice(None), slice(2, -2), slice(2, -2))
    hdr = vacio.header_for(prob)
    vacio.write_ascii(tmp_path / "in.ini", hdr, vacio.positions(prob)[inner], prob.w[inner])
    p2 = vacio.problem_from_vac(tmp_path / "in.ini", ghosts="pad")
    assert p2.n == prob.n and np.allclose(p2.dx, prob.dx) and np.allclose(p2.xmin, prob.xmin)
    assert np.array_equal(p2.w, prob.w)


@pytest.mark.skipif(not REF_CONFIGS.is_dir(), reason="reference sources not present")
def test_reference_orszag_tang_tiles(tmp_path):
    """The reference's 2x2-tiled Orszag-Tang configuration (126^2 per tile):
    read every tile, assemble the 252^2 grid (tile i + 2 j at x-block i,
    y-block j), and check it against the vortex's uniform density and the
    grid spacing 1/252."""
    tiles = [vacio.read_ascii(REF_CONFIGS / f"zero1_ot_asc_252_np0202_00{k}.ini") for k in range(4)]
    for h, _, _ in tiles:
        assert (h["it"], h["t"], h["ndim"], h["nw"], h["n"]) == (0, 0.0, 2, 10, (126, 126))
        assert abs(h["eqpar"][0] - 5.0 / 3.0) < 1e-5
    w = np.block([[tiles[0][2], tiles[1][2]], [tiles[2][2], tiles[3][2]]])
    pos = np.block([[tiles[0][1], tiles[1][1]], [tiles[2][1], tiles[3][1]]])
    assert w.shape == (10, 252, 252)
    rho = 25.0 / (36.0 * np.pi)
    assert np.allclose(w[0], rho, rtol=1e-10)
    assert np.allclose(np.diff(pos[0], axis=1), 1.0 / 252, rtol=1e-8)
    assert np.allclose(np.diff(pos[1], axis=0), 1.0 / 252, rtol=1e-8)
    vacio.write_ascii(tmp_path / "ot252.ini", tiles[0][0], pos, w)
    prob = vacio.problem_from_vac(tmp_path / "ot252.ini", ghosts="pad")
    assert prob.n == (256, 256) and abs(prob.gamma - 5.0 / 3.0) < 1e-5
