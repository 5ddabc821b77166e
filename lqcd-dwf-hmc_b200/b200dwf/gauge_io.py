"""Gauge-configuration files of the benchmark driver, read and written on
the host and handed to the device as lexical Field_G arrays (the layout
`DomainWall.set_config`, `StoutSmear.set_config` and the HMC take).

Formats (file:line in the reference tree):
  Text_4x4x4x8  FieldIO_Text_4x4x4x8::read_file
                (src/lib/IO/fieldIO_Text_4x4x4x8.cpp:21-150): one number per
                line, per site of a 4x4x4x8 lattice (x fastest), per direction
                mu, the 18 reals of U_mu; tiled periodically onto the run's
                lattice.  The reference cannot write this format.
  Binary        FieldIO_Binary (src/lib/IO/fieldIO_Binary.cpp:22-176) with
                IO_Format::Gauge::ILDG_Format (src/lib/IO/io_format_gauge.h:
                35-60): per lexical site the four links' 18 reals, mu slowest
                within the site, as big-endian doubles.  Binary_Parallel
                (fieldIO_Binary_Parallel.cpp:36-160) writes the same bytes
                through MPI-IO on more than one rank.

The lexical Field_G array is Field(18, Nvol, 4): index r + 18 * (site +
Nvol * mu), site = x + Lx * (y + Ly * (z + Lz * t)).
"""
import numpy as np

TEXT_LATTICE = (4, 4, 4, 8)


def _check_lattice(lattice):
    lattice = [int(v) for v in lattice]
    if len(lattice) != 4 or min(lattice) < 1:
        raise ValueError("lattice must be four positive extents")
    return lattice


def read_text_4x4x4x8(path, lattice):
    """GaugeConfig("Text_4x4x4x8").read: the 4x4x4x8 file tiled onto lattice."""
    return tile_text_4x4x4x8(np.loadtxt(path, dtype=np.float64, ndmin=1), lattice, path)


def tile_text_4x4x4x8(vals, lattice, name="configuration"):
    """The numbers of a Text_4x4x4x8 file (site-major [t][z][y][x][mu][18])
    tiled periodically onto lattice, as the lexical Field_G(Nvol, 4)."""
    lx, ly, lz, lt = _check_lattice(lattice)
    nf = int(np.prod(TEXT_LATTICE))
    vals = np.asarray(vals, dtype=np.float64).reshape(-1)
    if vals.size < nf * 4 * 18:
        raise ValueError("%s: %d numbers, %d needed for a 4x4x4x8 configuration"
                         % (name, vals.size, nf * 4 * 18))
    f = vals[:nf * 72].reshape(TEXT_LATTICE[3], TEXT_LATTICE[2], TEXT_LATTICE[1],
                                TEXT_LATTICE[0], 4, 18)          # [t][z][y][x][mu][r]
    t = np.arange(lt) % TEXT_LATTICE[3]
    z = np.arange(lz) % TEXT_LATTICE[2]
    y = np.arange(ly) % TEXT_LATTICE[1]
    x = np.arange(lx) % TEXT_LATTICE[0]
    tiled = f[np.ix_(t, z, y, x)]                                # [t][z][y][x][mu][r]
    return np.ascontiguousarray(np.moveaxis(tiled, 4, 0)).reshape(-1)


def write_binary(path, u_lex, lattice):
    """GaugeConfig("Binary").write_file (the bytes Binary_Parallel writes)."""
    nvol = int(np.prod(_check_lattice(lattice)))
    u = np.asarray(u_lex, dtype=np.float64)
    if u.size != 72 * nvol:
        raise ValueError("configuration has %d reals, %d expected" % (u.size, 72 * nvol))
    ildg = np.ascontiguousarray(u.reshape(4, nvol, 18).transpose(1, 0, 2))
    ildg.astype(">f8").tofile(path)


def read_binary(path, lattice):
    """GaugeConfig("Binary").read: big-endian ILDG-ordered file -> Field_G."""
    nvol = int(np.prod(_check_lattice(lattice)))
    raw = np.fromfile(path, dtype=">f8")
    if raw.size != 72 * nvol:
        raise ValueError("%s: %d reals, %d expected" % (path, raw.size, 72 * nvol))
    return np.ascontiguousarray(raw.reshape(nvol, 4, 18).transpose(1, 0, 2)).astype(np.float64).reshape(-1)


def to_device(u_lex):
    """Upload a lexical Field_G array to the current CUDA device (float64)."""
    import torch
    return torch.from_numpy(np.ascontiguousarray(u_lex, dtype=np.float64)).cuda()


def from_device(u_dev):
    """Device configuration back to a host array for write_binary."""
    return u_dev.detach().to("cpu").numpy().reshape(-1)
