"""IO_rot's output layout as raw binary files (pip_b200.output): datasets, order and
dimensions of save_coordinates / write_time / save_varfiles, per-rank hyperslab writes of a
decomposed run (create_write_dataspaces), config.txt (mk_config) and restart.  CPU only."""
import numpy as np
import pytest

from decomp_cases import make_case
from pip_b200 import decomp, ics, output


def test_round_trip_and_order(tmp_path):
    s, Uh, Um = ics.kelvin_helmholtz(32, 16)          # flag_ir: ion and rec are written
    path = output.write_output(str(tmp_path), 3, s, 0.125, Uh, Um)
    assert path.endswith("t0003.bin")
    d = output.read_output(path)
    names = [ln.split()[0] for ln in open(str(tmp_path / "t0003.idx"))]
    assert names == ["xgrid", "ygrid", "zgrid", "dx", "dy", "dz", "time",
                     "ro_p", "mx_p", "my_p", "mz_p", "en_p", "bx", "by", "bz", "ion", "rec",
                     "ro_n", "mx_n", "my_n", "mz_n", "en_n"]
    x, y, z, dx, dy, dz = s.coordinates()
    for name, arr in zip(output.GRID, (x, y, z, dx, dy, dz)):
        assert np.array_equal(d[name], arr)
    assert d["time"] == 0.125
    ix, jx, kx = s.shape
    for n, name in enumerate(output.VAR_M[:8]):
        assert d[name].shape == (kx, jx, ix) and np.array_equal(d[name][0], Um[n])
    for n, name in enumerate(output.VAR_H):
        assert np.array_equal(d[name][0], Uh[n])
    ion, rec = output.ir_rates(s, Um)
    assert np.array_equal(d["ion"][0], ion) and np.array_equal(d["rec"][0], rec)
    # Fortran order: x fastest, the file bytes are the planes as laid out in memory
    raw = np.fromfile(path, dtype="<f8")
    off = int([ln.split()[2] for ln in open(str(tmp_path / "t0003.idx")) if ln.startswith("bx ")][0]) // 8
    assert np.array_equal(raw[off: off + ix * jx], Um[5].reshape(-1))


def test_ps_written_with_dedner(tmp_path):
    s, Uh, Um = ics.orszag_tang(16)
    d = output.read_output(output.write_output(str(tmp_path), 0, s, 0.0, Uh, Um))
    assert "ps" in d and "ion" not in d and np.array_equal(d["ps"][0], Um[8])


@pytest.mark.parametrize("case,world", [("ot", 2), ("ot", 4), ("kh", 2), ("bw", 4)])
def test_rank_hyperslabs_make_the_global_file(tmp_path, case, world):
    s, Uh, Um = make_case(case)
    ref = output.write_output(str(tmp_path / "one"), 1, s, 0.5, Uh, Um)
    out = str(tmp_path / "ranks")
    output.create_output(out, 1, s, 0.5)
    for r in reversed(range(world)):                 # any order of the ranks' writes
        b = decomp.block_of(s, world, r)
        output.write_output_block(out, 1, s, b, decomp.scatter(s, Uh, world, r),
                                  decomp.scatter(s, Um, world, r))
    assert open(ref, "rb").read() == open(output.file_stem(out, 1) + ".bin", "rb").read()
    assert open(ref[:-4] + ".idx").read() == open(output.file_stem(out, 1) + ".idx").read()


def test_alpha_c_dataset(tmp_path):
    """flag_col 2..7: def_varfiles' "ac" opens the variables; restart reads it back; the
    ranks' hyperslabs of it make the single writer's file."""
    s, Uh, Um = ics.orszag_tang(16, flag_col=5)
    ac = np.random.default_rng(2).random(Uh.shape[1:]) + 1.0
    with pytest.raises(ValueError, match="ac"):
        output.write_output(str(tmp_path / "x"), 0, s, 0.0, Uh, Um)
    ref = output.write_output(str(tmp_path / "one"), 2, s, 0.5, Uh, Um, ac)
    names = [ln.split()[0] for ln in open(ref[:-4] + ".idx")]
    assert names[7:9] == ["ac", "ro_p"]
    assert np.array_equal(output.read_output(ref)["ac"][0], ac)
    assert np.array_equal(output.restart_alpha_c(str(tmp_path / "one"), 2, s), ac)
    assert output.restart_alpha_c(str(tmp_path / "one"), 2, s.overrides(flag_col=1)) is None
    out = str(tmp_path / "ranks")
    output.create_output(out, 2, s, 0.5)
    for r in range(4):
        b = decomp.block_of(s, 4, r)
        output.write_output_block(out, 2, s, b, decomp.scatter(s, Uh, 4, r),
                                  decomp.scatter(s, Um, 4, r), decomp.scatter(s, ac[None], 4, r)[0])
    assert open(ref, "rb").read() == open(output.file_stem(out, 2) + ".bin", "rb").read()


def test_config_and_restart(tmp_path):
    s, Uh, Um = ics.orszag_tang(16)
    text = "2.0d0          :gm_d;\n1.0d-8         :ro_lim;\n# no key here\n"
    output.mk_config(str(tmp_path), s, text)
    lines = open(str(tmp_path / "config.txt")).read().splitlines()
    assert lines[:3] == ["gm_d:2.0d0", "ro_lim:1.0d-8", "ENDSETTING"]
    cfg = output.read_config(str(tmp_path))
    assert (cfg["nvar_h"], cfg["nvar_m"]) == (5, 9) and tuple(cfg["margin"]) == s.margin
    assert tuple(cfg["shape"]) == s.shape and cfg["gm"] == s.gm and cfg["flag_bnd"] == s.flag_bnd
    output.write_output(str(tmp_path), 7, s, 0.25, Uh, Um)
    t, h, m = output.restart(str(tmp_path), 7, s)
    assert t == 0.25 and np.array_equal(h, Uh) and np.array_equal(m, Um)
    with pytest.raises(ValueError):
        output.restart(str(tmp_path), 7, s.overrides(flag_divb=0))
    with pytest.raises(ValueError):
        output.restart(str(tmp_path), 7, s.overrides(ix0=32, jx0=32))
