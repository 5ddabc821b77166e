"""Host-side pieces of bench.py's JSON line, on the CPU: the algorithmic
bytes and flops per half-site it divides by (the fused D_eo of the
operator's own count), and the name of the dagger-hop kernel the roofline
reports, read from the library's tuning table."""
import os
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

import bench  # noqa: E402


def test_bytes_and_flops_per_half_site():
    # Ls = 16, FP64: 24 reals in and out per slice, 8 links of 18 reals
    assert bench.BYTES_PER_HALF_SITE == 16 * 24 * 16 + 8 * 18 * 8 == 7296
    assert bench.FLOPS_PER_HALF_SITE == 1488 * 16 == 23808
    assert abs(bench.FLOPS_PER_HALF_SITE / bench.BYTES_PER_HALF_SITE - 3.263) < 1e-3


def test_dagger_hop_kernel_name(monkeypatch):
    import b200dwf
    table = ("vh=331776 ls=16 prec=f64 epi=2 fk=0 variant=0 us=797.0\n"
             "vh=331776 ls=16 prec=f64 epi=1 fk=0 variant=3 us=805.0\n"
             "vh=65536 ls=16 prec=f64 epi=1 fk=0 variant=0 us=140.0\n")
    monkeypatch.setattr(b200dwf, "tuning_table", lambda: table)
    assert bench.dagger_hop_kernel(331776).startswith("dwf_hop_tma_kernel<16,f64,EPI_DDAGEO>")
    assert "variant 3" in bench.dagger_hop_kernel(331776)
    assert bench.dagger_hop_kernel(65536).startswith("dwf_hop_kernel<16,f64,EPI_DDAGEO>")
    assert "EPI_DDAGEO" in bench.dagger_hop_kernel(1234)        # not tuned: generic name
