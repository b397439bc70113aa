"""Host-side readers (params, HKL, orientation, cache files) with the
reference's parsing semantics, and the synthetic generators."""
import numpy as np

from lauematching_b200 import formats, params as P, synth


def test_params_first_key_and_sscanf_prefix_semantics():
    txt = ("LatticeParameter 0.5 0.5 0.7 90 90 120 # comment\n"
           "NrPxX 1024\nNrPxY 512junk\n"          # %d reads the digit prefix
           "PxX 2e-4\nPxY 0.0002\n"
           "MinNrSpots abc\n"                      # failed conversion keeps the default
           "MinIntensity 12.5\n"
           "tol_c_over_a 0.01\ntol_LatC 1 1 1 0 0 0\n"   # c/a tolerance zeroes tol_LatC
           "R_Array 1 2\n"                         # partial read keeps the third value
           "UnknownKey 3\n"
           "ForwardFile /tmp/x.bin trailing\n"
           "Optimizer NelderMeadX\n")
    p = P.parse_params_text(txt)
    assert p.lattice == [0.5, 0.5, 0.7, 90.0, 90.0, 120.0]
    assert (p.nr_px_x, p.nr_px_y) == (1024, 512)
    assert p.min_nr_spots == 5 and p.min_intensity == 12.5
    assert p.tol_latc == [0.0] * 6 and p.tol_c_over_a == 0.01
    assert p.r_array == [1.0, 2.0, 0.0]
    assert p.forward_file == "/tmp/x.bin"
    assert p.optimizer == "NelderMead"
    assert "UnknownKey" in p.extra


def test_params_per_binary_defaults_and_fatal_checks():
    base = "LatticeParameter 0.3 0.3 0.3 90 90 90\nNrPxX 10\nNrPxY 10\n"
    assert P.parse_params_text(base, "cpu").batch_size == 1000000
    st = P.parse_params_text(base + "ResultDir out\nMinGoodSpots 3\n", "stream")
    assert (st.result_dir, st.min_good_spots) == ("out", 3)
    assert P.parse_params_text(base + "ResultDir out\n", "gpu").result_dir == "results_stream"
    for bad in ("LatticeParameter 0.3 0.3 0.3 90 90 90\n", "NrPxX 10\nNrPxY 10\n"):
        try:
            P.parse_params_text(bad)
        except P.ParamsError:
            continue
        raise AssertionError("fatal check missing")


def test_params_lines_longer_than_fgets_buffer_split():
    p = P.parse_params_text("LatticeParameter 0.3 0.3 0.3 90 90 90\nNrPxX 10\nNrPxY 10\n"
                            "X" * 1500 + "MinNrSpots 9\n")
    assert p.min_nr_spots == 5  # the key starts mid-line: never seen as a line start
    p = P.parse_params_text("LatticeParameter 0.3 0.3 0.3 90 90 90\nNrPxX 10\nNrPxY 10\n"
                            "X" * 998 + "\nMinNrSpots 9\n")
    assert p.min_nr_spots == 9


def test_hkl_reader_line_semantics(tmp_path):
    f = tmp_path / "h.csv"
    f.write_text("1 1 1 3\n2 0\n\n-2 2 0 8\n")
    h = formats.read_hkls(str(f))
    assert h.tolist() == [[1, 1, 1], [2, 0, 0], [0, 0, 0], [-2, 2, 0]]


def test_orientation_and_cache_round_trip(tmp_path):
    om = synth.shoemake_orientations(10, seed=4)
    formats.write_orientations(str(tmp_path / "o.bin"), om)
    with open(tmp_path / "o.bin", "ab") as f:
        f.write(b"\0" * 40)  # trailing partial record is ignored (size // 72)
    assert np.array_equal(formats.read_orientations(str(tmp_path / "o.bin")), om)
    rec = np.arange(10 * 7, dtype=np.uint16).reshape(10, 7)
    formats.write_forward_cache(str(tmp_path / "c.bin"), rec[5:], offset_records=5)
    formats.write_forward_cache(str(tmp_path / "c.bin"), rec[:5])
    assert np.array_equal(formats.read_forward_cache(str(tmp_path / "c.bin"), 10, 3), rec)


def test_shoemake_rotations_are_proper_and_counter_based():
    om = synth.shoemake_orientations(1000, seed=9).reshape(-1, 3, 3)
    assert np.allclose(om @ om.transpose(0, 2, 1), np.eye(3), atol=1e-12)
    assert np.allclose(np.linalg.det(om), 1.0)
    part = synth.shoemake_orientations(10, seed=9, start=500).reshape(-1, 3, 3)
    assert np.array_equal(part, om[500:510])


def test_hexagonal_fundamental_zone():
    om = synth.shoemake_orientations(2000, seed=3)
    fz = synth.hexagonal_fundamental_zone(om)
    R = fz.reshape(-1, 3, 3)
    assert np.allclose(R @ R.transpose(0, 2, 1), np.eye(3), atol=1e-9)
    q = synth._om_to_quat(fz)
    s = synth._HEX_SYM / np.linalg.norm(synth._HEX_SYM, axis=1, keepdims=True)
    w = np.abs(s[None, :, 0] * q[:, None, 0] - (s[None, :, 1:] * q[:, None, 1:]).sum(-1))
    assert np.all(w[:, 0] >= w.max(1) - 1e-9)  # identity is the best representative
    # same crystal orientation: input and reduced rotations differ by one of the
    # 622 operators, whose rotation angles are 0, 60, 120 or 180 degrees
    q0 = synth._om_to_quat(om)
    ang = np.degrees(2 * np.arccos(np.clip(np.abs((q0 * q).sum(1)), 0, 1)))
    assert np.all(np.min(np.abs(ang[:, None] - np.array([0, 60, 120, 180])), axis=1) < 0.01)


def test_hkl_generators():
    fcc = synth.hkls_cubic(8)
    assert len(fcc) == 1240
    f2 = (fcc.astype(np.int64) ** 2).sum(1)
    assert np.all(np.diff(f2) >= 0)
    assert np.all(((fcc[:, 0] + fcc[:, 1]) % 2 == 0) & ((fcc[:, 1] + fcc[:, 2]) % 2 == 0))
    assert len(synth.hkls_hexagonal(10)) == 7790
