"""Dataset readers (glc.datasets and include/glc_io.hpp): the reference driver's text and raw
binary readers and the SOSD layout, on temporary files (no GPU)."""
import os
import subprocess

import numpy as np
import pytest

from glc import datasets as D

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_text_reader(tmp_path):
    p = tmp_path / "v.txt"
    p.write_text("  12\n\n-7\t\nabc\n9000000000\n  3  \n")
    assert D.read_text_file(str(p), np.int64).tolist() == [12, -7, 9000000000, 3]
    assert D.read_text_file(str(tmp_path / "missing.txt")) is None


def test_binary_and_sosd_readers(tmp_path):
    v = np.arange(1000, dtype=np.uint64) * np.uint64(3) + np.uint64(1 << 60)
    p = tmp_path / "v.bin"
    v.tofile(p)
    assert np.array_equal(D.read_binary_file(str(p), np.uint64), v)
    (tmp_path / "odd.bin").write_bytes(b"\x00" * 7)
    assert D.read_binary_file(str(tmp_path / "odd.bin"), np.uint32) is None
    s = tmp_path / "v.sosd"
    D.write_sosd_file(str(s), v)
    assert np.array_equal(D.read_sosd_file(str(s), np.uint64), v)
    (tmp_path / "bad.sosd").write_bytes(np.array([5], "<u8").tobytes() + b"\x00" * 16)
    assert D.read_sosd_file(str(tmp_path / "bad.sosd"), np.uint64) is None


def test_cpp_readers_compile_and_agree(tmp_path):
    src = tmp_path / "io.cpp"
    src.write_text(r'''
#include "glc_io.hpp"
#include <cstdio>
int main(int argc, char** argv) {
  std::vector<long long> t; std::vector<unsigned long long> b, s;
  if (!read_text_file(argv[1], t) || !read_binary_file(argv[2], b) || !read_sosd_file(argv[3], s)) return 1;
  std::vector<unsigned int> bad;
  if (read_binary_file(argv[4], bad)) return 2;
  unsigned long long sum = 0;
  for (auto x : t) sum += (unsigned long long)x;
  for (auto x : b) sum += x;
  for (auto x : s) sum += x;
  printf("%zu %zu %zu %llu\n", t.size(), b.size(), s.size(), sum);
  return 0;
}
''')
    exe = tmp_path / "io"
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-I" + os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    (tmp_path / "t.txt").write_text("5\n-2\n\n x\n7\n")
    v = np.arange(10, dtype=np.uint64)
    v.tofile(tmp_path / "b.bin")
    D.write_sosd_file(str(tmp_path / "s.sosd"), v * np.uint64(2))
    (tmp_path / "odd.bin").write_bytes(b"\x00" * 6)
    out = subprocess.run([str(exe), str(tmp_path / "t.txt"), str(tmp_path / "b.bin"), str(tmp_path / "s.sosd"),
                          str(tmp_path / "odd.bin")], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    assert out.stdout.split() == ["3", "10", "10", str(5 - 2 + 7 + 45 + 90)]
