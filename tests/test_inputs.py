"""Input layer (host only): .de.bin files, the GPU bench's data modes and the
DLATMS spectrum-prescribed cache, each against the reference's format and
formulas (gpu/bench/tridiag_dc_bench.cu:229-447,
cpu/jobs/run_spectrum_de_cache_job.sh:52-110)."""
import math
import os

import numpy as np
import pytest
from scipy.linalg import lapack

import build as brdc_build
from brdc import inputs


@pytest.fixture(scope="module", autouse=True)
def _built():
    brdc_build.build()


# ---------------------------------------------------------------- .de.bin

def test_de_compact_roundtrip(tmp_path):
    rng = np.random.default_rng(5)
    d, e = rng.standard_normal(37), rng.standard_normal(36)
    p = str(tmp_path / "a.de.bin")
    inputs.write_de(p, d, e)
    assert os.path.getsize(p) == 8 + (2 * 37 - 1) * 8
    assert int(np.fromfile(p, dtype="<i8", count=1)[0]) == 37
    d2, e2 = inputs.read_de(p)
    assert np.array_equal(d, d2) and np.array_equal(e, e2)


def test_de_order_one(tmp_path):
    p = str(tmp_path / "one.de.bin")
    inputs.write_de(p, [3.5], [])
    d, e = inputs.read_de(p)
    assert d.tolist() == [3.5] and e.size == 0


def test_de_dense_payload(tmp_path):
    # dense payload: column-major n x n, D = A(i,i), E = A(i+1,i)
    n = 9
    rng = np.random.default_rng(6)
    a = rng.standard_normal((n, n))  # a[row, col]
    p = str(tmp_path / "dense.de.bin")
    with open(p, "wb") as f:
        f.write(np.asarray([n], dtype="<i8").tobytes())
        f.write(np.asfortranarray(a).tobytes(order="F"))
    d, e = inputs.read_de(p)
    assert np.array_equal(d, np.array([a[i, i] for i in range(n)]))
    assert np.array_equal(e, np.array([a[i + 1, i] for i in range(n - 1)]))


@pytest.mark.parametrize("n, payload", [(0, 0), (-3, 8), (5, 7 * 8), (5, 10 * 8)])
def test_de_rejects_bad_files(tmp_path, n, payload):
    p = str(tmp_path / "bad.de.bin")
    with open(p, "wb") as f:
        f.write(np.asarray([n], dtype="<i8").tobytes())
        f.write(b"\0" * payload)
    with pytest.raises(ValueError):
        inputs.read_de(p)


def test_de_rejects_short_header_and_bad_shapes(tmp_path):
    p = str(tmp_path / "short.de.bin")
    with open(p, "wb") as f:
        f.write(b"\1\2\3")
    with pytest.raises(ValueError):
        inputs.read_de(p)
    with pytest.raises(FileNotFoundError):
        inputs.read_de(str(tmp_path / "missing.de.bin"))
    with pytest.raises(ValueError):
        inputs.write_de(str(tmp_path / "x.de.bin"), np.ones(4), np.ones(4))


# ------------------------------------------------------- GPU bench modes

def _mt19937_raw(seed, count):
    # numpy's own MT19937 with the classic init_genrand seeding, an
    # implementation independent of the C++ library's std::mt19937
    bg = np.random.MT19937(0)
    bg._legacy_seeding(seed)
    return bg.random_raw(count).astype(np.uint64)


def _mt19937_64_raw(seed, count):
    # MT19937-64 (Matsumoto & Nishimura), parameters of std::mt19937_64
    mask = (1 << 64) - 1
    nn, mm = 312, 156
    mt = [seed & mask]
    for i in range(1, nn):
        mt.append((6364136223846793005 * (mt[-1] ^ (mt[-1] >> 62)) + i) & mask)
    out, idx = [], nn
    upper, lower = (mask << 31) & mask, (1 << 31) - 1
    for _ in range(count):
        if idx >= nn:
            for i in range(nn):
                x = (mt[i] & upper) | (mt[(i + 1) % nn] & lower)
                xa = (x >> 1) ^ (0xB5026F5AA96619E9 if x & 1 else 0)
                mt[i] = mt[(i + mm) % nn] ^ xa
            idx = 0
        y = mt[idx]
        idx += 1
        y ^= (y >> 29) & 0x5555555555555555
        y ^= (y << 17) & 0x71D67FFFEDA60000 & mask
        y ^= (y << 37) & 0xFFF7EEE000000000 & mask
        y ^= y >> 43
        out.append(y)
    return out


def test_mt19937_64_restatement():
    # the 10000th output of a default-seeded (5489) mt19937_64 is fixed by
    # the C++ standard
    assert _mt19937_64_raw(5489, 10000)[-1] == 9981545732273789042


def _canonical32(raw):
    # generate_canonical<double, 53> over a 32-bit engine: two draws,
    # (x0 + x1 2^32) / 2^64
    x0, x1 = raw[0::2].astype(np.float64), raw[1::2].astype(np.float64)
    return (x0 + x1 * 4294967296.0) / 18446744073709551616.0


@pytest.mark.parametrize("n, index", [(1, 0), (2, 0), (100, 3), (1000, 1)])
def test_bench_mode_matches_independent_engine(n, index):
    d, e = inputs.generate("bench", n, index)
    c = _canonical32(_mt19937_raw(1234 + index, 2 * (2 * n - 1)))
    assert np.array_equal(d, (float(n) + 0.25 * np.arange(n)) + (c[:n] * 1.0 + (-0.5)))
    assert np.array_equal(e, c[n:] * (0.95 - 0.05) + 0.05)


@pytest.mark.parametrize("n", [1, 3, 64])
def test_test_mode_matches_independent_engine(n):
    d, e = inputs.generate("test", n)
    v = _canonical32(_mt19937_raw(1300 + n, 2 * n * n)).reshape(n, n) * 2.0 + (-1.0)  # [col, row]
    assert np.array_equal(d, np.diagonal(v) + n)
    assert np.array_equal(e, np.diagonal(v, 1))


@pytest.mark.parametrize("n", [1, 5, 300])
def test_paper_uniform_matches_independent_engine(n):
    seed = ((n * 0x9E3779B97F4A7C15) & ((1 << 64) - 1)) ^ 0x94D049BB133111EB
    raw = _mt19937_64_raw(seed, 2 * n - 1)
    c = np.array([min(float(x) / 18446744073709551616.0, math.nextafter(1.0, 0.0)) for x in raw])
    d, e = inputs.generate("uniform", n)
    assert np.array_equal(d, c[:n] * 2.0 + (-1.0))
    assert np.array_equal(e, c[n:] * (0.30 - 0.10) + 0.10)


@pytest.mark.parametrize("n", [1, 2, 257])
def test_paper_closed_forms(n):
    d, e = inputs.generate("toeplitz", n)
    assert np.all(d == 2.0) and np.all(e == 0.25) and e.size == n - 1
    d, e = inputs.generate("clustered", n)
    c = 0.5 * (n + 1.0)
    assert d.tolist() == [1.0 + 1.0e-12 * ((i + 1) - c) for i in range(n)]
    assert e.tolist() == [1.0e-4 * (1.0 + 0.1 * math.cos(0.33 * (i + 1))) for i in range(n - 1)]


def test_paper_normal_shape():
    d, e = inputs.generate("normal", 4001)
    d2, e2 = inputs.generate("normal", 4001)
    assert np.array_equal(d, d2) and np.array_equal(e, e2)
    assert np.all(e >= 0.0)
    assert abs(d.mean()) < 0.1 and abs(d.std() - 1.0) < 0.05
    assert abs(e.mean() - 0.2 * math.sqrt(2.0 / math.pi)) < 0.01


def test_generate_rejects():
    with pytest.raises(ValueError):
        inputs.generate("dense", 8)
    with pytest.raises(ValueError):
        inputs.generate("bench", 0)


# -------------------------------------------------- spectrum-prescribed cache

@pytest.mark.parametrize("mode", ["uniform", "normal", "clustered"])
def test_dlatms_spectrum(mode):
    n = 512
    d, e, info, eig = inputs.spectrum_case(mode, n)
    assert info == 0 and d.size == n and e.size == n - 1
    w = lapack.dsterf(d, e)[0]
    assert np.max(np.abs(np.sort(eig) - w)) < 1e-13 * np.max(np.abs(w))
    d2, e2, _, _ = inputs.spectrum_case(mode, n)
    assert np.array_equal(d, d2) and np.array_equal(e, e2)
    if mode == "clustered":
        # MODE 1, COND 1e12: one eigenvalue of modulus 1, the rest 1e-12
        a = np.sort(np.abs(eig))
        assert a[-1] == 1.0 and np.all(a[:-1] == 1.0e-12)
    elif mode == "uniform":
        # MODE 6 draws the spectrum from DIST and does not rescale it
        assert np.all((eig > 0.0) & (eig < 1.0))


def test_spectrum_toeplitz_and_cache(tmp_path):
    d, e, info, eig = inputs.spectrum_case("toeplitz", 64)
    assert info == 0 and eig is None and np.all(d == 2.0) and np.all(e == 0.25)
    lines = inputs.write_spectrum_cache(str(tmp_path), sizes=(128, 200), out=None)
    assert lines[0] == "mode,n,path,generator,info"
    assert len(lines) == 1 + 4 * 2
    for ln in lines[1:]:
        mode, n, path, gen, info = ln.split(",")
        assert info == "0" and os.path.exists(path)
        assert gen == ("structured_toeplitz" if mode == "toeplitz" else "dlatms_symmetric_band")
        d, e = inputs.read_de(path)
        d0, e0, _, _ = inputs.spectrum_case(mode, int(n))
        assert np.array_equal(d, d0) and np.array_equal(e, e0)


def test_cli_generate(tmp_path):
    p = str(tmp_path / "g.de.bin")
    assert inputs._main(["generate", "bench", "33", p, "--index", "2"]) == 0
    d, e = inputs.read_de(p)
    d0, e0 = inputs.generate("bench", 33, 2)
    assert np.array_equal(d, d0) and np.array_equal(e, e0)
