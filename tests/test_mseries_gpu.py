"""The benchmark driver's random numbers drawn on the device
(b200_rng_*: RandomNumbers_parallel<RandomNumbers_Mseries>) against the
reference corelib's own draws: the uniform stream bit for bit, the Gaussians
to the last bits of the device's log/sqrt/sin/cos, across consecutive calls
(the streams advance) and after a reset; and against the CPU restatement on
a lattice of the benchmark's plane count."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "mseries_parallel.npz")
TOL = 1e-14       # absolute, on numbers of order 1 (Box-Muller through device libm)


def test_device_generator_matches_reference():
    import torch
    import b200dwf
    g = np.load(GOLD)
    meta = json.loads(str(g["meta"]))
    lat, ls, seed = meta["lattice"], meta["Ls"], meta["seed"]
    r = b200dwf.MseriesParallel(lat, seed)
    u = r.uniform_lex_global(2, 1).cpu().numpy()
    h = r.gauss_lex_global(8, 4).cpu().numpy()
    x = r.gauss_lex_global(24, ls).cpu().numpy()
    r.reset(seed + 1)
    h2 = r.gauss_lex_global(8, 4).cpu().numpy()
    torch.cuda.synchronize()
    assert np.array_equal(u, g["u"])
    for got, ref in ((h, g["h"]), (x, g["x"]), (h2, g["h2"])):
        assert np.abs(got - ref).max() < TOL


def test_device_generator_matches_oracle_other_shapes():
    """Odd extents, a block that does not fill the last 32-number step, and
    many planes: device against the CPU restatement."""
    import b200dwf
    from oracle.mseries import MseriesParallel as Oracle
    lat, seed = [2, 3, 5, 6], 987
    dev = b200dwf.MseriesParallel(lat, seed)
    ora = Oracle(lat, seed)
    for nin, nex in ((2, 3), (6, 1), (24, 2)):
        got = dev.gauss_lex_global(nin, nex).cpu().numpy()
        ref = ora.gauss_lex_global(nin, nex)
        assert np.abs(got - ref).max() < TOL, (nin, nex)
    got = dev.uniform_lex_global(3, 2).cpu().numpy()
    assert np.array_equal(got, ora.uniform_lex_global(3, 2))


def test_rejects_odd_gaussian_blocks():
    import b200dwf
    r = b200dwf.MseriesParallel([2, 2, 2, 2], 1)
    with pytest.raises(b200dwf.B200Error):
        r.gauss_lex_global(3, 1)


def test_refuses_seeds_past_the_int_delay():
    """Plane zt starts from the delay (seed + 1) Lz Lt + zt, an int in the
    reference (randomNumbers_parallel_Mseries.cpp:52-55); seeds that push it
    past INT_MAX are refused at create and reset, the largest one that fits
    is taken (Lz Lt = 2048: seed <= 1048574)."""
    import b200dwf
    with pytest.raises(b200dwf.B200Error, match="seed too large"):
        b200dwf.MseriesParallel([2, 2, 32, 64], 1234578)
    r = b200dwf.MseriesParallel([2, 2, 32, 64], 1048574)
    with pytest.raises(b200dwf.B200Error, match="seed too large"):
        r.reset(1048575)


def _set_ip_su3(h, nvol):
    """Langevin_Momentum::set_iP_SU3 (src/lib/HMC/langevin_Momentum.cpp:171-209)
    on Field(8, Nvol, 4) Gaussians -> lexical Field_G iP."""
    h = h.reshape(4 * nvol, 8)
    sq3r = 1.0 / np.sqrt(3.0)
    c = [h[:, k] for k in range(8)]
    ip = np.zeros((4 * nvol, 18))
    cols = {1: c[2] + c[7] * sq3r, 2: c[1], 3: c[0], 4: c[4], 5: c[3], 6: -c[1], 7: c[0],
            9: -c[2] + c[7] * sq3r, 10: c[6], 11: c[5], 12: -c[4], 13: c[3], 14: -c[6],
            15: c[5], 17: -c[7] * 2.0 * sq3r}
    for k, v in cols.items():
        ip[:, k] = v
    return ip.reshape(-1)


def test_mseries_noise_heatbath_fields():
    """The HMC heatbath source on the generator: momenta built from the
    reference's draws as set_iP_SU3 does, pseudofermion noise = the even sites
    of the reference's lexical draw (Index_eo order), delivered to the
    operator's device field without a host copy."""
    import torch
    import b200dwf
    from b200dwf.hmc import MseriesNoise
    g = np.load(GOLD)
    meta = json.loads(str(g["meta"]))
    lat, ls, seed = meta["lattice"], meta["Ls"], meta["seed"]
    nvol = int(np.prod(lat))
    noise = MseriesNoise(lat, seed)
    noise.rng.uniform_lex_global(2, 1)          # the fixture's first draw
    ip = torch.zeros(18 * 4 * nvol, dtype=torch.float64, device="cuda")
    noise.momentum(ip)
    assert np.abs(ip.cpu().numpy() - _set_ip_su3(g["h"], nvol)).max() < 1e-13
    op = b200dwf.DomainWall(lat, ls, 0.1, 1.8)
    f = op.new_field(0)
    noise.fermion(f)
    lex = g["x"].reshape(ls, nvol, 24)
    nx, ny, nz, nt = lat
    ev = []
    for t in range(nt):
        for z in range(nz):
            for y in range(ny):
                for ix2 in range(nx // 2):
                    ev.append(2 * ix2 + ((y + z + t) & 1) + nx * (y + ny * (z + nz * t)))
    ref = lex[:, ev, :].reshape(-1)
    assert np.abs(op.reverse(f) - ref).max() < TOL


def test_trajectory_with_the_drivers_generator():
    """A device 2+1-flavour trajectory drawing its heatbath from the device
    generator equals the same trajectory fed, through HostNoise, with the
    fields the CPU restatement of the generator produces (momentum first,
    then each fermion action in registration order, as the reference's
    HMC_General::langevin consumes them)."""
    import torch
    from b200dwf.hmc import HostNoise, MseriesNoise
    from oracle.mseries import MseriesParallel as Oracle
    from test_hmc_nf2p1 import _hmc_from_meta, golden
    meta, u, _ = golden()
    lat, ls, seed = meta["lattice"], meta["Ls"], 4242
    nvol = int(np.prod(lat))
    ora = Oracle(lat, seed)
    ip_ref = _set_ip_su3(ora.gauss_lex_global(8, 4), nvol)
    nx, ny, nz, nt = lat
    e = np.arange(nvol // 2)
    ix2, yzt = e % (nx // 2), e // (nx // 2)
    y, z, t = yzt % ny, (yzt // ny) % nz, yzt // (ny * nz)
    even = 2 * ix2 + ((y + z + t) & 1) + nx * (y + ny * (z + nz * t))
    xis = [ora.gauss_lex_global(24, ls).reshape(ls, nvol, 24)[:, even, :].reshape(-1)
           for _ in range(3)]
    out = []
    for noise in (MseriesNoise(lat, seed), HostNoise(ip_ref, xis)):
        hmc = _hmc_from_meta(meta)
        ud = torch.from_numpy(u.copy()).cuda()
        hmc.set_config(ud)
        ip = torch.zeros_like(ud)
        h0, _ = hmc.langevin(ip, noise)
        hmc.integrator.evolve(meta["tau"], ip, ud)
        h1, _ = hmc.calc_hamiltonian(ip)
        out.append((h0, h1 - h0, ud.cpu().numpy()))
    assert out[0][0] == pytest.approx(out[1][0], rel=1e-13)
    assert abs(out[0][1] - out[1][1]) < 1e-8
    assert np.max(np.abs(out[0][2] - out[1][2])) < 1e-10
