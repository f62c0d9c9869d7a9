"""CPU tests of the C-ABI library: it loads, exports every symbol declared in
include/aces_b200.h, and its DPD metadata reproduces the reference's layout
(acescore/aces_com_symloc.F, aces_com_sympop.F) -- no GPU needed."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT
import acesb200 as ab
from acesb200.dpd import DPD, pair_kind


@pytest.fixture(scope="module")
def lib():
    return ab.load()


def test_exports_match_header(lib):
    hdr = open(os.path.join(ROOT, "include", "aces_b200.h")).read()
    declared = set(re.findall(r"^\s*(?:const char \*|double \*|long long |int )(\w+)\(", hdr, re.M))
    assert declared == set(ab.SYMBOLS)
    for name in declared:
        assert hasattr(lib.h, name), name


def test_dpd_counts_h2o(lib):
    # H2O/DZP C2v populations of out.zmat.035.ccsd; the reference prints
    # "Norm of T2AB vector (3087 symmetry allowed elements)" and
    # "Norm of T1AA vector (39 symmetry allowed elements)"
    lib.sym_init([3, 1, 1, 0], [10, 3, 6, 2])
    n_t2ab = sum(lib.irpdpd(h, 13) * lib.irpdpd(h, 14) for h in range(1, 5))
    assert n_t2ab == 3087
    assert lib.irpdpd(1, 9) == 39
    # a<b / i<j packed (types 1, 3) and a<=b (type 5)
    vrt = np.array([10, 3, 6, 2])
    assert lib.irpdpd(1, 1) == sum(n * (n - 1) // 2 for n in vrt)
    assert lib.irpdpd(1, 5) == sum(n * (n + 1) // 2 for n in vrt)
    assert lib.irpdpd(2, 13) == 2 * (10 * 3 + 6 * 2)
    assert ab.load().h.aces_dirprd(2, 3) == 4


def test_isymoff_offsets_h2o(lib):
    lib.sym_init([3, 1, 1, 0], [10, 3, 6, 2])
    # total irrep 2 (B2), FULL (a,b): blocks ordered by irrep of b
    vrt = [10, 3, 6, 2]
    off = 1
    for hq in range(4):
        hp = hq ^ 1
        assert lib.isymoff(hq + 1, 2, 13) == off
        off += vrt[hp] * vrt[hq]


def test_dpd_tables_cover_every_pair_once(lib):
    lib.sym_init([2, 1, 0, 1], [4, 2, 3, 1])
    irr_o = [0, 0, 1, 3]
    irr_v = [0, 0, 0, 0, 1, 1, 2, 2, 2, 3]
    d = DPD(lib, irr_o, irr_v)
    for t in (1, 3, 5, 9, 11, 13, 14, 18):
        idx, sgn, hpq = d.table(t)
        for h in range(4):
            stored = idx[(hpq == h) & (sgn == 1)]
            n = lib.irpdpd(h + 1, t)
            assert sorted(stored.tolist()) == list(range(n)), (t, h)
        if pair_kind(t)[2] == 1:   # a<b: diagonal pairs are not stored
            assert np.all(sgn[np.eye(*sgn.shape, dtype=bool)] == 0)


def test_records_roundtrip_host_only(lib):
    x = np.arange(7, dtype=np.float64) * 0.5
    lib.putrec("TESTREC", x)
    np.testing.assert_array_equal(lib.getrec("TESTREC", 7), x)
    assert lib.h.aces_reclen(b"TESTREC") == 56
    with pytest.raises(ab.AcesError):
        lib.getrec("NOSUCHREC", 1)
    with pytest.raises(ab.AcesError):
        lib.getrec("TESTREC", 8)


def test_bad_arguments_return_status(lib):
    assert lib.h.aces_sym_init(3, (ctypes.c_int * 3)(1, 1, 1), (ctypes.c_int * 3)(1, 1, 1)) < 0
    lib.sym_init([1], [1])
    assert lib.h.aces_irpdpd(2, 13) < 0
    assert lib.h.aces_irpdpd(1, 23) < 0
    assert lib.h.aces_getlst(None, 1, 1, 9, 1) < 0


@pytest.mark.parametrize("fn", ["aces_xgemm", "aces_xgemm_static"])
def test_xgemm_rejects_short_leading_dimensions(lib, fn):
    """DGEMM's argument checks (tools/xgemm.F passes them to DGEMM): lda below
    the rows of A as stored (m for 'N', k for 'T'), ldb below the rows of B
    (k for 'N', n for 'T') and ldc < m are refused before any device work, so
    this runs without a GPU; the pointers are never dereferenced."""
    f = getattr(lib.h, fn)
    extra = (ab.PREC_FP64,) if fn == "aces_xgemm" else ()
    m, n, k = 7, 5, 3
    bad = [  # transa, transb, lda, ldb, ldc
        (b"N", b"N", m - 1, k, m), (b"T", b"N", k - 1, k, m),
        (b"N", b"N", m, k - 1, m), (b"N", b"T", m, n - 1, m), (b"N", b"N", m, k, m - 1),
    ]
    for ta, tb, lda, ldb, ldc in bad:
        st = f(ta, tb, m, n, k, 1.0, None, lda, None, ldb, 0.0, None, ldc, *extra)
        assert st == -1, (ta, tb, lda, ldb, ldc)
    # m*n == 0: quick return before any check of the operands
    assert f(b"N", b"N", 0, n, k, 1.0, None, 1, None, k, 0.0, None, 1, *extra) == 0


def test_pool_stats_is_callable_without_a_gpu(lib):
    calls, mallocs, cached = lib.pool_stats()
    assert calls >= 0 and mallocs >= 0 and cached >= 0 and mallocs <= calls


def test_header_is_c99_and_config_layout_matches_ctypes(tmp_path):
    """include/aces_b200.h compiles as C99 (a Fortran/C host includes it as
    is), and the aces_cc_config layout a C compiler gives (size and every
    field offset) is the one acesb200.CCConfig passes through ctypes."""
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    fields = [f for f, _ in ab.CCConfig._fields_]
    src = tmp_path / "layout.c"
    body = "\n".join(f'  printf("%s %zu\\n", "{f}", offsetof(aces_cc_config, {f}));' for f in fields)
    src.write_text(
        "#include <stddef.h>\n#include <stdio.h>\n#include \"aces_b200.h\"\n"
        "int main(void) {\n"
        '  printf("sizeof %zu\\n", sizeof(aces_cc_config));\n' + body + "\n  return 0;\n}\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-pedantic", "-I",
                    os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True, capture_output=True, text=True)
    out = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True,
                                                       text=True, check=True).stdout.split("\n")
               if line)
    assert int(out["sizeof"]) == ctypes.sizeof(ab.CCConfig)
    for f in fields:
        assert int(out[f]) == getattr(ab.CCConfig, f).offset, f
    # the EOM config the same way
    efields = [f for f, _ in ab.EOMConfig._fields_]
    body = "\n".join(f'  printf("%s %zu\\n", "{f}", offsetof(aces_eom_config, {f}));'
                     for f in efields)
    src.write_text(
        "#include <stddef.h>\n#include <stdio.h>\n#include \"aces_b200.h\"\n"
        "int main(void) {\n"
        '  printf("sizeof %zu\\n", sizeof(aces_eom_config));\n' + body + "\n  return 0;\n}\n")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-pedantic", "-I",
                    os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True, capture_output=True, text=True)
    out = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True,
                                                       text=True, check=True).stdout.split("\n")
               if line)
    assert int(out["sizeof"]) == ctypes.sizeof(ab.EOMConfig)
    for f in efields:
        assert int(out[f]) == getattr(ab.EOMConfig, f).offset, f


def test_autotune_switch_and_stats_without_a_gpu(lib):
    """aces_set_autotune takes modes 0/1/2 only; with nothing tuned the stats
    are zero; the switch is left off (the default) for the other tests."""
    assert lib.h.aces_set_autotune(3) == -1
    assert lib.h.aces_set_autotune(-1) == -1
    lib.set_autotune(2)
    lib.set_autotune(1)
    assert lib.autotune_stats() == (0, 0, 0.0)
    lib.set_autotune(0)
    assert lib.autotune_stats() == (0, 0, 0.0)


def test_autotune_choices_save_and_load_without_a_gpu(lib, tmp_path):
    """Tile choices round-trip through their text file; a file with a choice
    the tuner could not make for its class (CTA pairs without the >= 256-row
    flag, a tile width on an unbatched product) is refused and loads
    nothing."""
    header = "# aces-b200 tile choices v1\n"
    rows = ("0 1 0 2 2 24 1 0 1 1\n"       # single product: no split K
            "0 1 1 8 2 10 2 0 0 1\n"       # single product >= 256 rows: CTA pairs
            "1 2 1 30 0 12 1 0 0 0\n"      # grouped launch of two products
            "2 4 7 40 2 20 1 256 0 0\n")   # batched FP32 output: 256-wide tiles
    lib.set_autotune(2)
    good = tmp_path / "choices.txt"
    good.write_text(header + rows)
    lib.autotune_load(good)
    assert lib.autotune_stats() == (4, 2, 0.0)
    out = tmp_path / "saved.txt"
    lib.autotune_save(out)
    assert out.read_text() == header + rows
    for bad_row in ("0 1 0 2 2 24 2 0 0 1\n", "0 1 1 8 2 10 1 256 0 0\n", "3 1 0 1 1 1 1 0 0 0\n",
                    "0 1 0 2 2 24 1 0 1\n"):
        bad = tmp_path / "bad.txt"
        bad.write_text(header + bad_row)
        with pytest.raises(ab.AcesError):
            lib.autotune_load(bad)
        assert lib.autotune_stats()[0] == 4
    notfile = tmp_path / "other.txt"
    notfile.write_text("0 1 0 2 2 24 1 0 1 1\n")
    with pytest.raises(ab.AcesError):
        lib.autotune_load(notfile)
    with pytest.raises(ab.AcesError):
        lib.autotune_load(tmp_path / "missing.txt")
    lib.set_autotune(2)
    assert lib.autotune_stats() == (0, 0, 0.0)
