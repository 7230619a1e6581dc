"""CPU tests of the native file formats (host-only entry points of the C ABI):
text catalogues (src/input_formats.f90:227-333) against numpy's text reader,
the result table (src/main.f90:699-702), and the binary marks stream
(src/input_formats.f90:528-603) against the oracle's numpy restatement in both
directions."""
import numpy as np
import pytest


def write_table(path, a, comments=True):
    with open(path, "w") as f:
        if comments:
            f.write("# x y ...\n\n")
        for i, row in enumerate(a):
            sep = "," if i % 7 == 3 else " "
            f.write(sep.join(repr(float(v)) if i % 2 else f"{v:.9e}" for v in row) + "\n")
            if i % 97 == 5:
                f.write("   \n")


def test_shape_catalogue_and_mask(tpcf, tmp_path):
    rng = np.random.default_rng(1)
    a = rng.normal(size=(5003, 7)).astype(np.float32)
    a[:, 5] = rng.uniform(-0.2, 1.0, 5003).astype(np.float32)  # w <= 0 rows dropped
    p = tmp_path / "shapes.txt"
    write_table(p, a)
    S = tpcf.load_standard_shape_catalog(p)
    keep = a[:, 5] > 0
    for k, col in zip(("x", "y", "z", "e1", "e2", "w", "m"), range(7)):
        np.testing.assert_array_equal(getattr(S, k), a[keep, col])


def test_lens_catalogue_masks(tpcf, tmp_path):
    rng = np.random.default_rng(2)
    a = rng.normal(size=(2000, 5)).astype(np.float32)
    p = tmp_path / "lenses.txt"
    np.savetxt(p, a, fmt="%.9g")
    L = tpcf.load_standard_lens_catalog(p)
    keep = (a[:, 4] > 0) & (a[:, 2] >= 0)
    np.testing.assert_array_equal(L.val, a[keep, 3])
    L2 = tpcf.load_standard_lens_catalog(p, apply_masks=False)
    np.testing.assert_array_equal(L2.x, a[:, 0])
    K = tpcf.load_standard_kappa_map(p)
    np.testing.assert_array_equal(K.kappa_B, a[a[:, 4] > 0, 3])


def test_decimal_rounding_matches_numpy(tpcf, tmp_path):
    rng = np.random.default_rng(3)
    txt = rng.uniform(-1e3, 1e3, (400000, 2))
    p = tmp_path / "big.txt"
    np.savetxt(p, txt, fmt="%.17g")
    got = tpcf.read_table(p, 2)
    np.testing.assert_array_equal(got.T, txt.astype(np.float32))


def test_thread_counts_agree_across_chunk_boundaries(tpcf, tmp_path):
    # ~1.5 MB, so up to ~20 threads get a piece; pieces start and end among
    # comment lines, blank lines, CRLF endings and '+' signs, and the last line
    # has no newline.  Every thread count must give the rows in file order.
    rng = np.random.default_rng(7)
    a = rng.normal(size=(30000, 5)).astype(np.float32)
    lines = []
    for i, row in enumerate(a):
        if i % 101 == 0:
            lines.append("# comment " + str(i))
        if i % 37 == 0:
            lines.append("")
        txt = " ".join(("+" if (i + k) % 11 == 0 and v >= 0 else "") + f"{v:.9g}" for k, v in enumerate(row))
        lines.append(txt + ("\r" if i % 13 == 0 else ""))
    p = tmp_path / "mixed.txt"
    p.write_bytes("\n".join(lines).encode())
    keep = (a[:, 4] > 0) & (a[:, 2] >= 0)
    ref = None
    for nt in (1, 3, 8, 20):
        got = tpcf.read_table(p, 5, keep_positive_col=4, keep_nonnegative_col=2, n_threads=nt)
        np.testing.assert_array_equal(got.T, a[keep])
        if ref is None:
            ref = got
        np.testing.assert_array_equal(got, ref)


def test_malformed_line_is_an_error(tpcf, tmp_path):
    p = tmp_path / "bad.txt"
    p.write_text("1 2 3\n4 5\n")
    with pytest.raises(tpcf.TPCFError):
        tpcf.read_table(p, 3)
    # a bad line in the last of several threads' pieces
    big = tmp_path / "bad_late.txt"
    big.write_text("1 2 3\n" * 200000 + "4 5\n" + "6 7 8\n" * 10)
    with pytest.raises(tpcf.TPCFError):
        tpcf.read_table(big, 3, n_threads=8)


def test_result_table(tpcf, tmp_path):
    nb = 6
    r = type("R", (), {})()
    r.theta = np.linspace(0.1, 1.0, nb).astype(np.float32)
    r.g_t, r.g_x = np.float32([1e-3] * nb), np.float32([-2e-4] * nb)
    r.weights = np.float32([5.0] * nb)
    r.n_pairs = np.arange(nb, dtype=np.int64) * 10 ** 10
    r.mean_theta = r.theta * np.float32(1.01)
    p = tmp_path / "xi.txt"
    tpcf.write_result_table(p, r, spherical_coords=True)
    t = np.loadtxt(p)
    assert t.shape == (nb, 6)
    np.testing.assert_allclose(t[:, 0], np.degrees(r.theta.astype(np.float64)), rtol=1e-6)
    np.testing.assert_array_equal(t[:, 4], r.n_pairs)
    np.testing.assert_allclose(t[:, 1], r.g_t, rtol=1e-7)


def test_marks_stream_round_trips(tpcf, oracle, tmp_path):
    rng = np.random.default_rng(4)
    fields = []
    for n, nb in ((300, 7), (0, 7), (1000, 7)):
        fields.append({"x": rng.normal(size=n), "y": rng.normal(size=n), "w": rng.uniform(0, 2, n),
                       "xi_E": rng.normal(size=(n, nb)), "xi_B": rng.normal(size=(n, nb)),
                       "K": rng.uniform(size=(n, nb))})
    p1, p2 = tmp_path / "a.bin", tmp_path / "b.bin"
    oracle.marks_write(p1, fields)
    got = tpcf.load_survey_marks(p1)
    assert len(got) == 3
    for g, f in zip(got, fields):
        for k in ("x", "y", "w", "xi_E", "xi_B", "K"):
            np.testing.assert_array_equal(getattr(g, k), np.asarray(f[k], np.float32))
    tpcf.save_marks(p2, got)
    assert p1.read_bytes() == p2.read_bytes()
    back = oracle.marks_read(p2)
    np.testing.assert_array_equal(back[2]["K"], np.asarray(fields[2]["K"], np.float32))


def test_marks_header_is_checked(tpcf, tmp_path):
    p = tmp_path / "bad.bin"
    p.write_bytes(np.zeros(200, np.int64).tobytes())
    with pytest.raises(tpcf.TPCFError):
        tpcf.load_survey_marks(p)
