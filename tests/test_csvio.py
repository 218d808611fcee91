"""CPU tests of qaf.csvio, the reader/writer of the reference's physical-field
CSV files (field_visual / file_init): the writer's text equals what a C++
output stream writes for the same doubles, and the reader inverts it to the
6 significant digits the format keeps."""
import os
import subprocess

import numpy as np
import pytest

from qaf import csvio

VALUES = np.array([[0.0, 1.0, -2.5e-7, 123456789.0, 0.1],
                   [-0.333333333333, 1e-300, 7.0e22, -1.0, 2.0 / 3.0],
                   [5e-5, -0.0, 42.0, 1.5e-12, -987654.321]])


CXX_WRITER = r"""
#include <fstream>
#include <cstdio>
int main(int argc, char** argv) {
    // one line per row, every value followed by a comma, the stream's default format
    std::ofstream out(argv[1]);
    int ny, nx;
    std::FILE* in = std::fopen(argv[2], "rb");
    if (std::fread(&ny, sizeof(int), 1, in) != 1 || std::fread(&nx, sizeof(int), 1, in) != 1) return 1;
    for (int j = 0; j < ny; ++j) {
        for (int i = 0; i < nx; ++i) {
            double v;
            if (std::fread(&v, sizeof(double), 1, in) != 1) return 1;
            out << v << ",";
        }
        out << std::endl;
    }
    std::fclose(in);
    return 0;
}
"""


def test_writer_matches_a_cpp_output_stream(tmp_path):
    src = tmp_path / "w.cpp"
    src.write_text(CXX_WRITER)
    exe = tmp_path / "w"
    subprocess.run(["g++", "-O1", "-o", str(exe), str(src)], check=True)
    raw = tmp_path / "v.bin"
    with open(raw, "wb") as f:
        np.array(VALUES.shape, dtype=np.int32).tofile(f)
        VALUES.astype(np.float64).tofile(f)
    subprocess.run([str(exe), str(tmp_path / "cpp.csv"), str(raw)], check=True)
    csvio.write_field(str(tmp_path / "py.csv"), VALUES)
    assert (tmp_path / "py.csv").read_bytes() == (tmp_path / "cpp.csv").read_bytes()


def test_reader_inverts_the_writer_to_six_digits(tmp_path):
    rng = np.random.default_rng(3)
    a = rng.standard_normal((12, 16)) * 10.0 ** rng.integers(-8, 8, (12, 16))
    p = str(tmp_path / "f.csv")
    csvio.write_field(p, a)
    b = csvio.read_field(p, nx=16, ny=12)
    assert b.shape == (12, 16)
    assert np.array_equal(b, np.vectorize(lambda v: float("%g" % v))(a))
    assert np.all(np.abs(b - a) <= 5e-6 * np.abs(a))


def test_reader_takes_lines_without_trailing_commas(tmp_path):
    p = tmp_path / "f.csv"
    p.write_text("1,2,3\n4,5,6\n")
    assert np.array_equal(csvio.read_field(str(p)), [[1, 2, 3], [4, 5, 6]])


def test_reader_errors(tmp_path):
    p = str(tmp_path / "f.csv")
    csvio.write_field(p, np.zeros((4, 6)))
    with pytest.raises(ValueError):
        csvio.read_field(p, nx=4, ny=6)        # the reference's "size not match!"
    with pytest.raises(FileNotFoundError):
        csvio.read_field(str(tmp_path / "missing.csv"))
    (tmp_path / "ragged.csv").write_text("1,2,\n3,\n")
    with pytest.raises(ValueError):
        csvio.read_field(str(tmp_path / "ragged.csv"))


def test_nonfinite_values_print_as_the_cpp_stream_does(tmp_path):
    assert csvio.format_value(float("inf")) == "inf"
    assert csvio.format_value(float("-inf")) == "-inf"
    assert csvio.format_value(float("nan")) in ("nan", "-nan")
