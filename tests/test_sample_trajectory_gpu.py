"""The reference's published single-GPU trajectory, reproduced on the device.

sample_1gpu/ of the reference (HMC_DWF_Nf2p1_eo.yaml, main.yaml, run.log):
8^4 lattice from conf_04040408.txt tiled periodically, Moebius domain-wall
fermions b=1.5, c=0.5, M0=1.0, Ls=12; Nf1 = 0.02 as a rational ratio over
Pauli-Villars (16 poles in the force, 24 in the heatbath and Hamiltonian),
light 0.0005 over Hasenbusch 0.002 over Pauli-Villars 1.0; tree-level
Symanzik gauge action beta=4.17 (c_plaq 5/3, c_rect -1/12); 3 stout steps
rho=0.1; Omelyan [2,1,3] on levels [0,0,1,2], length 0.1; the
Mseries_parallel generator reset to i_conf = 200000 (hmc_dwf_eo.cpp:399);
solver tolerances |r|^2/|b|^2 < 1e-28, multishift 1e-26 (MD) and 1e-28
(calcH); the reference's own rational tables.  Published:
H_total(init) = 1003485.4326439571, H(diff) = 0.00083995 (from the two
totals, 0.0008399482), plaq(final) = 0.622916188574 (run.log:1557-2000).

tests/golden/sample_8x8x8x8.npz holds the configuration file's numbers, the
table files and the published values with their log lines (written by
tests/golden/make_golden.py sample)."""
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def fixture():
    z = np.load(os.path.join(HERE, "golden", "sample_8x8x8x8.npz"))
    return (json.loads(str(z["meta"])), z["conf_04040408"], json.loads(str(z["tables"])),
            json.loads(str(z["published"])))


def links(meta, conf):
    from b200dwf.gauge_io import tile_text_4x4x4x8
    return tile_text_4x4x4x8(conf, meta["lattice"])


def plaquette(u, lattice):
    """Average Re tr of the plaquettes / 3 over sites and the 6 planes."""
    lx, ly, lz, lt = lattice
    v = lx * ly * lz * lt
    c = u.reshape(4, v, 18)
    m = (c[..., 0::2] + 1j * c[..., 1::2]).reshape(4, lt, lz, ly, lx, 3, 3)
    axis = {0: 4, 1: 3, 2: 2, 3: 1}
    tot = 0.0
    for mu in range(4):
        for nu in range(mu + 1, 4):
            umu, unu = m[mu], m[nu]
            unu_xmu = np.roll(unu, -1, axis=axis[mu] - 1)
            umu_xnu = np.roll(umu, -1, axis=axis[nu] - 1)
            p = umu @ unu_xmu @ np.conj(np.swapaxes(umu_xnu, -1, -2)) @ np.conj(np.swapaxes(unu, -1, -2))
            tot += np.trace(p, axis1=-2, axis2=-1).real.sum()
    return tot / (3.0 * 6.0 * v)


# ------------------------------------------------------------------ CPU

def test_fixture_links_and_initial_plaquette():
    """The tiled configuration is SU(3) and its plaquette is the published
    plaq(init) (run.log:1559) to the log's 12 digits."""
    meta, conf, _, pub = fixture()
    u = links(meta, conf)
    m = u.reshape(-1, 18)
    a = (m[:, 0::2] + 1j * m[:, 1::2]).reshape(-1, 3, 3)
    eye = np.einsum("nij,nkj->nik", a, np.conj(a))
    assert np.abs(eye - np.eye(3)).max() < 1e-12
    assert abs(np.linalg.det(a) - 1).max() < 1e-12
    assert plaquette(u, meta["lattice"]) == pytest.approx(pub["plaq_init"], abs=6e-13)


def test_fixture_tables_read_by_the_loader(tmp_path):
    """The reference's shipped Remez tables parse with this package's
    Math_Rational-format reader and meet the error each states."""
    from b200dwf.rational import read_table, max_rel_error
    _, _, tables, _ = fixture()
    assert len(tables) == 6
    for name, text in tables.items():
        (tmp_path / name).write_text(text)
        ne, de, lo, hi, err, a0, b, c = read_table(str(tmp_path / name))
        assert (lo, hi) == (1e-4, 10.0)
        # evaluating the sum in double precision rounds at a few 1e-14
        assert max_rel_error(a0, b, c, lo, hi, ne / de) <= max(1.05 * err, 5e-14)


# ------------------------------------------------------------------ GPU

@pytest.mark.gpu
def test_published_trajectory(tmp_path):
    import time
    import torch
    from b200dwf.hmc import build_dwf_nf2p1, MseriesNoise
    meta, conf, tables, pub = fixture()
    for name, text in tables.items():
        (tmp_path / name).write_text(text)
    c = meta
    hmc = build_dwf_nf2p1(c["lattice"], c["Ls"], c["M0"],
                          dict(l=c["mq_l"], h=c["mq_h"], s=c["mq_s"], pv=c["mq_pv"]),
                          c["beta"], c["c_plaq"], c["c_rect"], c["rho"], c["nsmear"],
                          c["nstep"], c["level"], c["tau"], c["lam"], c["nprec"], c["np_md"],
                          c["np_h"], (c["rat_lo"], c["rat_hi"]), c["tol_cg"], c["tol_cg"],
                          b=c["b"], c=c["c"], rational_dir=str(tmp_path),
                          tol2_rat_md=c["tol_ms_md"], tol2_rat_h=c["tol_ms_h"])
    u0 = links(meta, conf)
    ud = torch.from_numpy(u0.copy()).cuda()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    r = hmc.trajectory(ud, MseriesNoise(c["lattice"], c["seed"]))
    torch.cuda.synchronize()
    sec = time.perf_counter() - t0
    h0, dh = r["H0"], r["dH"]
    parts = [float(x) for x in r["parts0"]]
    plaq = plaquette(ud.cpu().numpy(), c["lattice"])
    print("SAMPLE_TRAJECTORY " + json.dumps(dict(H0=h0, dH=dh, parts0=parts, plaq_final=plaq,
                                                 seconds=sec, published=pub)))
    # the published start, per action (run.log:1523-1557)
    assert h0 == pytest.approx(pub["H_total_init"], abs=2e-7)
    for got, key in zip(parts[1:], ("H_Frational_init", "H_Fratio_Nf2_init", "H_Fratio_Nf2prec_init",
                                "H_Grectangle_init")):
        assert got == pytest.approx(pub[key], abs=2e-8 * abs(pub[key]) + 1e-8), key
    # the published end: the three reference builds agree on H(diff) to 6e-9
    dh_pub = pub["H_total_final"] - pub["H_total_init"]
    assert abs(dh - dh_pub) < 5e-8, (dh, dh_pub)
    assert round(dh, 8) == pytest.approx(pub["H_diff"], abs=1.01e-8)
    assert plaq == pytest.approx(pub["plaq_final"], abs=6e-13)
