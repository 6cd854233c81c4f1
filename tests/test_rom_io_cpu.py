"""Dense ROM files (host code of the C-ABI library, no GPU): the reference's Matrix Market
reader / writer and solution table (test/krylovTestGPU/matrixInSingleLoop/gpu/src/io/io.cu,
src/tools/AuxiliaryFunctions.cpp:80-110)."""
import numpy as np
import pytest

from staccato_b200 import rom_io


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint64)


def test_round_trip_is_bit_exact(tmp_path):
    rng = np.random.default_rng(0)
    A = (rng.standard_normal((37, 19)) * 10.0 ** rng.integers(-300, 300, (37, 19))
         + 1j * rng.standard_normal((37, 19)))
    A[0, 0] = complex(-0.0, 5e-324)          # signed zero, smallest subnormal
    A[1, 2] = complex(np.inf, -np.inf)
    p = tmp_path / "a.mtx"
    rom_io.write_mtx_dense(str(p), A)
    B = rom_io.read_mtx_dense(str(p))
    assert B.shape == A.shape
    assert np.array_equal(_bits(B.real), _bits(A.real)) and np.array_equal(_bits(B.imag), _bits(A.imag))
    head = p.read_text().splitlines()[:3]
    assert head[0] == "%%MatrixMarket matrix coordinate complex dense column major"
    assert head[1] == "37\t19"
    assert len(head[2].split("\t")) == 2


def test_reads_reference_layout_with_comments_and_blank_tail(tmp_path):
    # banner, comment lines, tab separators, column order, trailing blank line
    text = ("%%MatrixMarket matrix coordinate complex dense column major\n% written by a test\n"
            "2\t3\n1.5\t-2\n3\t4\n5\t6\n7\t8\n9\t10\n11\t-12e-3\n\n")
    p = tmp_path / "k.mtx"
    p.write_text(text)
    A = rom_io.read_mtx_dense(str(p))
    ref = np.array([[1.5 - 2j, 5 + 6j, 9 + 10j], [3 + 4j, 7 + 8j, 11 - 0.012j]])
    assert np.array_equal(A, ref)


def test_reads_headerless_real_and_row_major_files(tmp_path):
    p = tmp_path / "plain.mtx"
    p.write_text("2 2\n1 0\n2 0\n3 0\n4 1\n")  # no banner: complex pairs, column order
    assert np.array_equal(rom_io.read_mtx_dense(str(p)), np.array([[1, 3], [2, 4 + 1j]]))
    p = tmp_path / "real.mtx"
    p.write_text("%%MatrixMarket matrix array real general\n2 3\n1\n2\n3\n4\n5\n6\n")
    assert np.array_equal(rom_io.read_mtx_dense(str(p)), np.array([[1, 3, 5], [2, 4, 6]], dtype=complex))
    p = tmp_path / "rm.mtx"
    p.write_text("%%MatrixMarket matrix coordinate complex dense row major\n2\t2\n1\t0\n2\t0\n3\t0\n4\t0\n")
    assert np.array_equal(rom_io.read_mtx_dense(str(p)), np.array([[1, 2], [3, 4]], dtype=complex))


@pytest.mark.parametrize("body", ["2 2\n1 0\n2 0\n3 0\n", "2 2\n1 0\n2 0\n3 0\n4 0\n5 0\n", "x y\n", ""])
def test_malformed_files_raise(tmp_path, body):
    p = tmp_path / "bad.mtx"
    p.write_text(body)
    with pytest.raises(rom_io.RomFileError):
        rom_io.read_mtx_dense(str(p))


def test_missing_file_raises(tmp_path):
    with pytest.raises(rom_io.RomFileError, match="cannot read"):
        rom_io.read_mtx_dense(str(tmp_path / "none.mtx"))


def test_solution_table_and_rom_triple(tmp_path):
    x = np.array([1.0 + 2.0j, -3.25e-17 + 0.1j, 7.0 - 0.0j])
    p = tmp_path / "solution_small.dat"
    rom_io.write_solution(str(p), x)
    raw = p.read_bytes()
    assert raw.startswith(b"Real" + b" " * 21 + b"    Imag") and b"\r\n" in raw
    assert np.array_equal(rom_io.read_solution(str(p)), x)
    rng = np.random.default_rng(1)
    K, M = rng.standard_normal((5, 5)) + 0j, rng.standard_normal((5, 5)) + 1j
    rom_io.write_mtx_dense(str(tmp_path / "K.mtx"), K)
    rom_io.write_mtx_dense(str(tmp_path / "M.mtx"), M)
    K2, M2, D2 = rom_io.load_rom(str(tmp_path), K="K.mtx", M="M.mtx")
    assert np.array_equal(K2, K) and np.array_equal(M2, M) and D2 is None
