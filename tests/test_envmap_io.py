"""Row a1: cubemap face extraction from a 4x3 cross, in the Python mirror and in the C++
shim (include/nwprt_engine.hpp), against Environment_Map's constructors
(EnvironmentMap.cpp:10-126): .npy and .hdr crosses are flipped vertically
(EnvironmentMap.cpp:96-101; HDRLoaderResult::get, Renderer/HDRloader.h:21-25), then cut
into faces +X,-X,+Y,-Y,-Z,+Z at the cells (2,1), (0,1), (1,2), (1,0), (1,1), (3,1) of the
flipped image (EnvironmentMap.cpp:117-122).

The test cross is S=4 (16 x 12 texels).  Every texel holds distinct values: R = its
row-major index in the file's image (row 0 = first row stored), G = its cell's index in
the file's image (cell row * 4 + cell column), B = 255 - R.  All are integers below 256,
which RGBE stores exactly."""
import os
import subprocess

import numpy as np
import pytest

from neural_wavelet_prt_demo_b200 import _lib
from neural_wavelet_prt_demo_b200.engine import EnvironmentMap, read_hdr
from tests.helpers import write_hdr

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
S = 4
H, W = 3 * S, 4 * S


def make_cross():
    r = np.arange(H * W, dtype=np.float32).reshape(H, W)
    cell = (np.arange(H)[:, None] // S) * 4 + (np.arange(W)[None, :] // S)
    return np.stack([r, cell.astype(np.float32), 255 - r], axis=-1)


def expected_faces(img):
    """Face f, texel (r, c) = the file image's row H-1-(cell_row*S + r), column cell_col*S + c."""
    cells = [(2, 1), (0, 1), (1, 2), (1, 0), (1, 1), (3, 1)]
    out = np.empty((6, S, S, 3), np.float32)
    for f, (cc, cr) in enumerate(cells):
        for r in range(S):
            for c in range(S):
                out[f, r, c] = img[H - 1 - (cr * S + r), cc * S + c]
    return out


def test_cross_layout_known_texels():
    faces = EnvironmentMap.cross_to_faces(make_cross())
    assert np.array_equal(faces, expected_faces(make_cross()))
    # +X texel (0,0): file row 7, column 8 -> R = 7*16 + 8; its cell is the file's (row 1, col 2)
    assert faces[0, 0, 0, 0] == 120 and np.all(faces[0, ..., 1] == 6)
    # +Y is the file's top-middle cell, -Y the bottom-middle one, -Z the centre, +Z the right
    assert np.all(faces[2, ..., 1] == 1) and np.all(faces[3, ..., 1] == 9)
    assert np.all(faces[4, ..., 1] == 5) and np.all(faces[5, ..., 1] == 7)
    assert np.all(faces[1, ..., 1] == 4)
    # -Y texel (0,0): the file's last row, column 4
    assert faces[3, 0, 0, 0] == (H - 1) * W + 4


@pytest.mark.parametrize("rle", [True, False])
def test_hdr_reader_round_trip(tmp_path, rle):
    img = make_cross()
    p = tmp_path / "x.hdr"
    write_hdr(p, img, rle)
    assert np.array_equal(read_hdr(str(p)), img)


def test_hdr_repeat_code_and_zero_exponent(tmp_path):
    # flat scanline: one pixel, then (1,1,1,3) repeats it three times; E=0 gives tiny values
    p = tmp_path / "r.hdr"
    row = bytes([10, 20, 30, 129, 1, 1, 1, 3])
    row2 = bytes([5, 6, 7, 0]) * 4
    p.write_bytes(b"#?RADIANCE\n\n-Y 2 +X 4\n" + row + row2)
    img = read_hdr(str(p))
    assert np.array_equal(img[0], np.tile(np.array([10, 20, 30], np.float32) / 128, (4, 1)))
    assert np.array_equal(img[1, 0], np.ldexp(np.array([5, 6, 7], np.float32) / 256, -128).astype(np.float32))


def test_hdr_reader_rejects_bad_files(tmp_path):
    p = tmp_path / "bad.hdr"
    p.write_bytes(b"#?RGBE\n\n-Y 1 +X 1\n" + bytes(4))
    with pytest.raises(RuntimeError):
        read_hdr(str(p))
    p.write_bytes(b"#?RADIANCE\n\n-Y 2 +X 1\n" + bytes(4))   # one scanline short
    with pytest.raises(RuntimeError):
        read_hdr(str(p))


def make_env_folder(tmp_path, name="room"):
    img = make_cross()
    d = tmp_path / "env"
    for sub in ("cube", "sh", "waveletcoeffs", "waveletstrength"):
        (d / sub).mkdir(parents=True)
    write_hdr(d / "cube" / (name + ".hdr"), img, rle=True)
    np.save(d / "sh" / (name + ".npy"), np.arange(81 * 3, dtype=np.float32).reshape(81, 3))
    np.save(d / "waveletcoeffs" / (name + ".npy"), np.array([5, 3, 90], np.int64))   # numpy's default int
    np.save(d / "waveletstrength" / (name + ".npy"), np.arange(9, dtype=np.float32).reshape(3, 3))
    return d, img


def test_python_folder_and_file_constructors(tmp_path):
    d, img = make_env_folder(tmp_path)
    em = EnvironmentMap.from_folder(str(d), "room")
    assert np.array_equal(em.faces, expected_faces(img))
    assert em.topWaveletCoefficients.tolist() == [5, 3, 90]
    assert em.topWaveletStrength.shape == (3, 3) and em.shCoefficients.shape == (81, 3)
    np.save(tmp_path / "cross.npy", img)
    assert np.array_equal(EnvironmentMap.from_file(str(tmp_path / "cross.npy")).faces, expected_faces(img))
    with pytest.raises(RuntimeError, match="Invalid Env map File Name"):
        EnvironmentMap.from_folder(str(d), "missing")
    with pytest.raises(RuntimeError, match="Folder"):
        EnvironmentMap.from_folder(str(d / "sh" / "room.npy"), "room")


CPP_DRIVER = r'''
#include <cstdio>
#include "nwprt_engine.hpp"
static void dump(const char* path, const std::vector<float>& v) {
  FILE* f = std::fopen(path, "wb");
  std::fwrite(v.data(), sizeof(float), v.size(), f);
  std::fclose(f);
}
int main(int argc, char** argv) {
  // argv: npy cross, rle hdr, flat hdr, env folder, out dir
  std::string out = argv[5];
  nwprt::Environment_Map a{std::string(argv[1])};
  nwprt::Environment_Map b{std::string(argv[2])};
  nwprt::Environment_Map c{std::string(argv[3])};
  nwprt::Environment_Map d{argv[4], "room"};
  dump((out + "/a.bin").c_str(), a.faces);
  dump((out + "/b.bin").c_str(), b.faces);
  dump((out + "/c.bin").c_str(), c.faces);
  dump((out + "/d.bin").c_str(), d.faces);
  std::printf("%d %d %d %d %zu %zu %zu\n", a.face_size, d.face_size, d.topWaveletCoefficients[2],
              (int)d.topWaveletStrength[8], d.topWaveletCoefficients.size(), d.shCoefficients.size(),
              d.topWaveletStrength.size());
  int errors = 0;
  try { nwprt::Environment_Map e{argv[4], "missing"}; } catch (const std::runtime_error&) { ++errors; }
  try { nwprt::Environment_Map e{std::string(argv[4]) + "/x.png"}; } catch (const std::runtime_error&) { ++errors; }
  try { nwprt::Environment_Map e{std::string(argv[4]) + "/sh/room.npy", true}; } catch (const std::runtime_error&) { errors += 100; }
  std::printf("%d\n", errors);
  return 0;
}
'''


def test_cpp_shim_constructors(tmp_path):
    d, img = make_env_folder(tmp_path)
    np.save(tmp_path / "cross.npy", img)
    write_hdr(tmp_path / "rle.hdr", img, rle=True)
    write_hdr(tmp_path / "flat.hdr", img, rle=False)
    src = tmp_path / "envio.cpp"
    src.write_text(CPP_DRIVER)
    exe = tmp_path / "envio"
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                        "-L", os.path.dirname(_lib.LIB_PATH), "-lnwprt",
                        "-Wl,-rpath," + os.path.dirname(_lib.LIB_PATH)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    run = subprocess.run([str(exe), str(tmp_path / "cross.npy"), str(tmp_path / "rle.hdr"),
                          str(tmp_path / "flat.hdr"), str(d), str(tmp_path)], capture_output=True, text=True)
    assert run.returncode == 0, run.stderr
    lines = run.stdout.split("\n")
    assert lines[0].split() == ["4", "4", "90", "8", "3", "243", "9"]
    assert lines[1].strip() == "2"
    want = expected_faces(img)
    for name in "abcd":
        got = np.fromfile(tmp_path / f"{name}.bin", np.float32).reshape(6, S, S, 3)
        assert np.array_equal(got, want), name
