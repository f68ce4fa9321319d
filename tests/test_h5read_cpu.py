"""The pure-Python HDF5 reader and the dump discovery of the replay module, without a GPU.

Real files: the reference's own HDF5 test data, written by h5pp/libhdf5 (the committed subset under
tests/golden/reference_h5 everywhere; all 57 SVD test matrices and the eigenproblem fixtures where the reference tree
is present).  Their content checks the parse: every SVD test matrix is a normalised two-site state (unit Frobenius
norm), and the eigenproblem fixtures satisfy A v = lambda v with their stored eigenpairs.
Synthetic files: tests/h5writer.py writes the structures those files do not contain (chunked layouts with shuffle,
deflate and fletcher32 filters, edge chunks, version-2 object headers, link-message groups, nested groups, variable-
length string attributes) and the reader must return exactly what was written.
"""
import glob
import hashlib
import json
import os

import numpy as np
import pytest

from dmrg_b200 import replay
from dmrg_b200.h5read import H5Dataset, H5File, H5FormatError, H5Group

import h5writer

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = os.path.join(HERE, "golden", "reference_h5")
REFERENCE = "/root/reference"


def test_committed_fixtures_intact():
    with open(os.path.join(FIXTURES, "manifest.json")) as fh:
        manifest = json.load(fh)
    assert len(manifest) == 12
    for name, meta in manifest.items():
        with open(os.path.join(FIXTURES, name), "rb") as fh:
            data = fh.read()
        assert len(data) == meta["bytes"] and hashlib.sha256(data).hexdigest() == meta["sha256"]


def svd_matrix_files():
    files = sorted(glob.glob(os.path.join(REFERENCE, "tests/svd/testmatrices/svdmatrix_*.h5")))
    return files or sorted(glob.glob(os.path.join(FIXTURES, "svdmatrix_*.h5")))


def test_reference_svd_matrices_are_normalised_states():
    files = svd_matrix_files()
    assert len(files) >= 7
    for p in files:
        with H5File(p) as f:
            assert f.root.keys() == ["svdmatrix"]
            d = f["svdmatrix"]
            assert isinstance(d, H5Dataset) and d.dtype == np.complex128 and len(d.shape) == 2
            A = d.read()
            assert A.shape == d.shape and np.all(np.isfinite(A))
            assert abs(np.linalg.norm(A) - 1.0) < 1e-11, p
            assert np.linalg.norm(A.imag) > 0  # the imaginary member is read, not dropped


def test_reference_svd_bench_file():
    """bench/svd/data/svd-failed.h5: groups svd_lapacke_<n> with A, S, U, V and MKL's attributes."""
    with H5File(os.path.join(FIXTURES, "svd-failed.h5")) as f:
        assert f.root.keys() == [f"svd_lapacke_{i}" for i in range(4)]
        g = f["svd_lapacke_0"]
        assert isinstance(g, H5Group)
        at = g.attrs
        assert (at["rows"], at["cols"], at["rank_max"], at["info"]) == (58, 58, 116, 1)
        assert at["threshold"] == np.finfo(np.float64).eps
        assert at["Intel-MKL-MajorVersion"] == 2019
        A = g["A"].read()
        assert A.shape == (58, 58) and A.dtype == np.complex128
        assert g["S"].read().shape == (56,) and g["U"].shape == (58, 56) and g["V"].shape == (56, 58)
        A1 = f["svd_lapacke_1/A"].read()
        assert A1.shape == (100, 25) and A1.dtype == np.float64
        # the real bench matrices are rank 20 with singular values 445.7 and 52.05 at the top
        s = np.linalg.svd(A1, compute_uv=False)
        assert abs(s[0] - 445.71435789) < 1e-6 and s[19] > 1e-8 > s[20]
        assert f["svd_lapacke_1/U"].shape == (0, 0)


@pytest.mark.parametrize("name", ["lapacke_matrix-1A.h5", "lapacke_matrix-1B.h5", "lapacke_matrix-2A.h5", "lapacke_matrix-2B.h5"])
def test_reference_eigenproblem_fixtures(name):
    """tests/testmatrices/lapacke_matrix-*.h5 hold a real symmetric matrix with the eigenpairs the reference's LAPACK
    computed, a state theta and its overlaps |<v_i|theta>|: A V = V diag(w), and the overlaps follow."""
    with H5File(os.path.join(FIXTURES, name)) as f:
        A, w, V = f["matrix"].read(), f["eigvals"].read().ravel(), f["eigvecs"].read()
        th, ov = f["theta"].read().ravel(), f["overlaps"].read().ravel()
    assert A.shape[0] == A.shape[1] == len(w) == V.shape[0] == th.size
    assert np.allclose(A, A.T, atol=1e-12 * np.abs(A).max())
    assert np.linalg.norm(A @ V - V * w) < 1e-8 * np.linalg.norm(A)
    assert np.allclose(np.sort(w), np.linalg.eigvalsh(A), atol=1e-8 * np.abs(w).max())
    assert th.dtype == np.complex128 and abs(np.linalg.norm(th) - 1) < 1e-12
    assert np.max(np.abs(np.abs(V.T @ th) - ov)) < 1e-12


def write(tmp_path, root, name="t.h5"):
    p = str(tmp_path / name)
    h5writer.write(p, root)
    return p


def test_layouts_filters_and_types_round_trip(tmp_path):
    rng = np.random.default_rng(3)
    Z = rng.standard_normal((37, 23)) + 1j * rng.standard_normal((37, 23))
    X = rng.standard_normal((5, 7, 11))
    I = rng.integers(-1000, 1000, size=(13, 9))
    F = rng.standard_normal(19).astype(np.float32)
    root = {
        "contig": Z,
        "compact": {"__data__": X[0], "__layout__": "compact"},
        "chunked": {"__data__": Z, "__layout__": "chunked", "__chunk__": (8, 8)},
        "deflate": {"__data__": X, "__layout__": "chunked", "__chunk__": (2, 4, 5), "__filters__": ("shuffle", "deflate")},
        "fletcher": {"__data__": I, "__layout__": "chunked", "__chunk__": (13, 4), "__filters__": ("deflate", "fletcher32")},
        "v2hdr": {"__data__": Z[:3], "__ohdr_v2__": True},
        "f32": F,
        "scalar": np.float64(2.5),
        "ints": I,
    }
    with H5File(write(tmp_path, root)) as f:
        assert np.array_equal(f["contig"].read(), Z)
        assert np.array_equal(f["compact"].read(), X[0])
        assert np.array_equal(f["chunked"].read(), Z)
        assert np.array_equal(f["deflate"].read(), X)
        assert np.array_equal(f["fletcher"].read(), I)
        assert np.array_equal(f["v2hdr"].read(), Z[:3])
        assert f["f32"].read().dtype == np.float32 and np.array_equal(f["f32"].read(), F)
        assert f["scalar"].shape == () and f["scalar"].read() == 2.5
        assert f["ints"].dtype == np.int64 and np.array_equal(np.asarray(f["ints"]), I)


def test_groups_links_and_attributes(tmp_path):
    names = [f"contraction_{i}" for i in range(12)]  # more links than one symbol-table node holds (8)
    root = {n: {"x": np.full(3, i, float)} for i, n in enumerate(names)}
    root["linked"] = {"__links__": True, "__attrs__": {"label": "compact links", "n": np.int64(4)},
                      "inner": {"deep": {"__data__": np.arange(6.0).reshape(2, 3), "__ohdr_v2__": True}}}
    root["__attrs__"] = {"truncation_lim": 1e-8, "svd_lib": "lapacke", "fixed": b"gesdd\x00\x00\x00"}
    with H5File(write(tmp_path, root)) as f:
        assert sorted(f.root.keys()) == sorted(names + ["linked"])
        for i, n in enumerate(names):
            assert np.array_equal(f[n]["x"].read(), np.full(3, i, float))
        assert np.array_equal(f["linked/inner/deep"].read(), np.arange(6.0).reshape(2, 3))
        assert f["/linked/inner"].name == "/linked/inner"
        assert f["linked"].attrs == {"label": "compact links", "n": 4}
        at = f.root.attrs
        assert at["truncation_lim"] == 1e-8 and at["svd_lib"] == "lapacke" and at["fixed"] == "gesdd"
        assert "linked/inner/deep" in f and "linked/nothing" not in f
        with pytest.raises(KeyError):
            f["contraction_0/x/y"]
        paths = [p for p, _ in f.visit()]
        assert "/linked/inner/deep" in paths and len(paths) == 2 * len(names) + 3


def test_not_hdf5_and_unsupported_features(tmp_path):
    p = tmp_path / "plain.bin"
    p.write_bytes(b"\x00" * 4096)
    with pytest.raises(H5FormatError):
        H5File(str(p))
    # a filter the reader does not implement (szip, id 4) must fail loudly rather than return raw bytes
    q = write(tmp_path, {"d": {"__data__": np.ones((4, 4)), "__layout__": "chunked", "__chunk__": (4, 4), "__filters__": ("deflate",)}})
    data = bytearray(open(q, "rb").read())
    i = data.find(bytes([1, 0, 0, 0, 0, 0, 1, 0]))  # filter record: id 1, name length 0, flags 0, 1 value
    assert i > 0
    data[i] = 4
    open(q, "wb").write(bytes(data))
    with H5File(q) as f, pytest.raises(H5FormatError, match="filter 4"):
        f["d"].read()


def contraction_group(rng, spin, chiL, chiR, D, cplx):
    def r(*s):
        a = rng.standard_normal(s)
        return a + 1j * rng.standard_normal(s) if cplx else a

    return {"mps": r(spin, chiL, chiR), "mpo": r(D, D, spin, spin), "envL": r(chiL, chiL, D), "envR": r(chiR, chiR, D)}


def test_contraction_dumps_order_and_layout(tmp_path):
    rng = np.random.default_rng(9)
    groups = {f"contraction_{i}": contraction_group(rng, 2, 3 + i, 4 + i, 3, i % 2 == 1) for i in (0, 1, 2, 10)}
    root = dict(groups)
    root["other"] = {"x": np.zeros(2)}
    got = replay.contraction_dumps(write(tmp_path, root))
    assert [g["name"] for g in got] == ["contraction_0", "contraction_1", "contraction_2", "contraction_10"]
    for g in got:
        src = groups[g["name"]]
        for k in ("mps", "mpo", "envL", "envR"):
            assert g[k].flags.f_contiguous and np.array_equal(g[k], src[k])
    # a dump holding raw column-major buffers under reversed dimensions is read back in the same layout
    rev = {"contraction_0": {k: np.ascontiguousarray(v.transpose()) for k, v in groups["contraction_10"].items()}}
    g = replay.contraction_dumps(write(tmp_path, rev, "rev.h5"))[0]
    for k in ("mps", "mpo", "envL", "envR"):
        assert np.array_equal(g[k], groups["contraction_10"][k])
    bad = {"contraction_0": dict(groups["contraction_0"], envR=rng.standard_normal((5, 5, 3)))}
    with pytest.raises(ValueError, match="do not form a contraction"):
        replay.contraction_dumps(write(tmp_path, bad, "bad.h5"))


def test_svd_dumps_layouts(tmp_path):
    rng = np.random.default_rng(4)
    A = rng.standard_normal((6, 4)) + 1j * rng.standard_normal((6, 4))
    U, S, VT = np.linalg.svd(A, full_matrices=False)
    root = {
        "svd_0": {"A_cplx": A, "U_cplx": U, "S": S, "VT_cplx": VT,
                  "__attrs__": {"rank_max": np.int64(3), "truncation_lim": 1e-10, "info": np.int64(0), "svd_lib": "lapacke"}},
        "svd-fail": {"A_real": A.real, "__attrs__": {"rank_max": np.int64(4), "truncation_lim": 1e-6, "info": np.int64(2)}},
        "svd_lapacke_1": {"A": A, "S": S, "V": VT, "__attrs__": {"rank_max": np.int64(4), "threshold": 1e-12}},
    }
    got = {e["name"]: e for e in replay.svd_dumps(write(tmp_path, root))}
    assert set(got) == {"svd_0", "svd-fail", "svd_lapacke_1"}
    assert got["svd_0"]["rank_max"] == 3 and got["svd_0"]["truncation_lim"] == 1e-10 and got["svd_0"]["info"] == 0
    assert np.array_equal(got["svd_0"]["A"], A) and np.array_equal(got["svd_0"]["S"], S) and np.array_equal(got["svd_0"]["VT"], VT)
    assert got["svd-fail"]["A"].dtype == np.float64 and got["svd-fail"]["info"] == 2
    assert got["svd_lapacke_1"]["truncation_lim"] == 1e-12 and np.array_equal(got["svd_lapacke_1"]["VT"], VT)
    over = replay.svd_dumps(write(tmp_path, root, "o.h5"), truncation_lim=1e-3)
    assert all(e["truncation_lim"] == 1e-3 for e in over)
    # the reference's test-matrix layout: one root dataset, the test's limit 1e-8
    e = replay.svd_dumps(os.path.join(FIXTURES, "svdmatrix_6.h5"))
    assert len(e) == 1 and e[0]["name"] == "svdmatrix" and e[0]["truncation_lim"] == 1e-8 and e[0]["A"].shape == (2, 8)
    # the reference's bench file: info = 1 / -13 marks its outputs as failed; the inputs are still replayable
    b = replay.svd_dumps(os.path.join(FIXTURES, "svd-failed.h5"))
    assert [x["name"] for x in b] == [f"svd_lapacke_{i}" for i in range(4)]
    assert [x["info"] for x in b] == [1, -13, -13, -13] and b[0]["truncation_lim"] == np.finfo(float).eps


def test_eig_dumps_layout(tmp_path):
    """The eigensolver bench's eigs.h5 layout (bench/eig/main.cpp:45-62): eigs-<n> groups with a complex mps, real
    mpo2/envL2/envR2 and the recorded solve's attributes."""
    rng = np.random.default_rng(12)
    g = contraction_group(rng, 4, 5, 6, 9, False)
    mps = g["mps"] + 1j * rng.standard_normal(g["mps"].shape)
    root = {f"eigs-{i}": {"mps": mps, "mpo2": g["mpo"], "envL2": g["envL"], "envR2": g["envR"],
                          "__attrs__": {"eval": 0.25 * i, "rnorm": 1e-13, "iter": np.int64(40), "mv": np.int64(321),
                                        "dims": np.array([4, 5, 6], dtype=np.int64), "size": np.int64(120)}} for i in (2, 0, 1)}
    root["eigs_other"] = {"x": np.zeros(1)}
    got = replay.eig_dumps(write(tmp_path, root, "eigs.h5"))
    assert [e["name"] for e in got] == ["eigs-0", "eigs-1", "eigs-2"]
    for i, e in enumerate(got):
        assert np.array_equal(e["mps"], mps) and np.array_equal(e["mpo2"], g["mpo"])
        assert np.array_equal(e["envL2"], g["envL"]) and np.array_equal(e["envR2"], g["envR"])
        assert e["envL2"].flags.f_contiguous and e["mpo2"].dtype == np.float64
        assert e["attrs"]["eval"] == 0.25 * i and e["attrs"]["dims"] == [4, 5, 6] and e["attrs"]["mv"] == 321


def test_layout_and_attribute_message_versions(tmp_path):
    """Layout messages version 1/2 (compact, contiguous, chunked) and version 4 (single chunk, filtered or not;
    implicit index), and attribute messages version 2 and 3: each read back exactly."""
    rng = np.random.default_rng(21)
    X = rng.standard_normal((9, 7))
    Z = rng.standard_normal((6, 5)) + 1j * rng.standard_normal((6, 5))
    root = {
        "v1_contig": {"__data__": X, "__layout_version__": 1},
        "v2_compact": {"__data__": X[:2], "__layout__": "compact", "__layout_version__": 2},
        "v1_chunked": {"__data__": Z, "__layout__": "chunked", "__chunk__": (4, 2), "__layout_version__": 1, "__filters__": ("deflate",)},
        "v4_single": {"__data__": X, "__layout__": "chunked", "__chunk__": X.shape, "__layout_version__": 4, "__index__": "single"},
        "v4_single_f": {"__data__": Z, "__layout__": "chunked", "__chunk__": Z.shape, "__layout_version__": 4, "__index__": "single",
                        "__filters__": ("shuffle", "deflate")},
        "v4_implicit": {"__data__": X, "__layout__": "chunked", "__chunk__": (4, 3), "__layout_version__": 4, "__index__": "implicit"},
        "attrs_v2": {"__data__": np.zeros(1), "__attrs__": {"rank_max": np.int64(7), "svd_lib": "lapacke"}, "__attr_version__": 2},
        "attrs_v3": {"__data__": np.zeros(1), "__attrs__": {"threshold": 1e-12, "dims": np.array([4, 5, 6])}, "__attr_version__": 3},
    }
    with H5File(write(tmp_path, root)) as f:
        assert np.array_equal(f["v1_contig"].read(), X)
        assert np.array_equal(f["v2_compact"].read(), X[:2])
        assert np.array_equal(f["v1_chunked"].read(), Z)
        assert np.array_equal(f["v4_single"].read(), X)
        assert np.array_equal(f["v4_single_f"].read(), Z)
        assert np.array_equal(f["v4_implicit"].read(), X)
        assert f["attrs_v2"].attrs == {"rank_max": 7, "svd_lib": "lapacke"}
        a3 = f["attrs_v3"].attrs
        assert a3["threshold"] == 1e-12 and np.array_equal(a3["dims"], [4, 5, 6])
