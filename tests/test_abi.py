"""The C ABI library without a GPU: it loads, exports every declared symbol, its config struct matches
the header, defaults match the reference's Configuration::default(), and the host mirror behaves like
the reference's API (builder, error variants)."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "pacmap.h")


def _declared_functions():
    with open(HEADER) as f:
        src = f.read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pacmap_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(lib):
    names = _declared_functions()
    assert "pacmap_fit_transform" in names and "pacmap_knn_exact" in names
    so = C.CDLL(lib._abi.LIB_PATH)
    missing = [n for n in names if not hasattr(so, n)]
    assert not missing, missing


def test_config_struct_layout_matches_header(lib):
    fields = [f[0] for f in lib._abi.Config._fields_]
    prog = "#include <stdio.h>\n#include <stddef.h>\n#include \"pacmap.h\"\nint main(void){\n"
    prog += 'printf("%zu\\n", sizeof(pacmap_config));\n'
    for f in fields:
        prog += f'printf("%zu\\n", offsetof(pacmap_config, {f}));\n'
    prog += "return 0;}\n"
    with tempfile.TemporaryDirectory() as td:
        src, exe = os.path.join(td, "layout.c"), os.path.join(td, "layout")
        with open(src, "w") as f:
            f.write(prog)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), src, "-o", exe], check=True)
        out = [int(v) for v in subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()]
    assert out[0] == C.sizeof(lib._abi.Config)
    assert out[1:] == [getattr(lib._abi.Config, f).offset for f in fields]


def test_config_defaults_match_reference(lib):
    # lib.rs:208-224 Configuration::default()
    c = lib._abi.lib().pacmap_config_default()
    assert c.embedding_dimensions == 2 and c.init_kind == 0 and c.pair_kind == 0
    assert c.mid_near_ratio == 0.5 and c.far_pair_ratio == 2.0 and c.learning_rate == 1.0
    assert list(c.num_iters) == [100, 100, 250] and c.approx_threshold == 8000
    assert not c.has_seed and not c.has_override_neighbors and not c.snapshots
    py = lib.Configuration()
    assert (py.embedding_dimensions, py.mid_near_ratio, py.far_pair_ratio, py.learning_rate, py.num_iters,
            py.approx_threshold) == (2, 0.5, 2.0, 1.0, (100, 100, 250), 8000)
    assert isinstance(py.initialization, lib.Initialization.Pca)
    assert isinstance(py.pair_configuration, lib.PairConfiguration.Generate)


def test_builder_like_reference(lib):
    # tests.rs:7-19 test_configuration_builder
    cfg = lib.Configuration.builder().initialization(lib.Initialization.Random(42)).learning_rate(0.8) \
        .num_iters((50, 50, 100)).build()
    assert cfg.embedding_dimensions == 2 and cfg.learning_rate == 0.8 and cfg.num_iters == (50, 50, 100)


def test_error_classes_cover_reference_variants(lib):
    for name in ["SampleSize", "InvalidNearestNeighborShape", "EmptyArrayMean", "Normal", "InvalidNeighborCount",
                 "InvalidFarPointCount", "EmptyArrayMinMax", "ZeroRange", "Pca", "KnnConstruction", "KnnReservation",
                 "MissingTransform"]:
        assert issubclass(getattr(lib, name), lib.PaCMapError)


def test_host_side_validation_without_device(lib):
    # The reference checks n > 1 before anything else (lib.rs:300-302); so does the library, before
    # it touches a device.
    with pytest.raises(lib.SampleSize):
        lib.fit_transform(np.zeros((1, 4), np.float32), lib.Configuration(initialization=lib.Initialization.Random(0)))
    idx, dist = lib.knn.find_k_nearest_neighbors(np.zeros((0, 128), np.float32), 5)
    assert idx.shape == (0, 0) and dist.shape == (0, 0)


@pytest.mark.skipif(os.path.exists("/dev/nvidia0"), reason="a GPU is present")
def test_no_device_is_an_error_not_a_fallback(lib):
    x = np.random.default_rng(0).normal(size=(50, 4)).astype(np.float32)
    with pytest.raises(lib.NoDevice):
        lib.fit_transform(x, lib.Configuration(initialization=lib.Initialization.Random(0)))
    with pytest.raises(lib.NoDevice):
        lib.knn.find_k_nearest_neighbors(x, 3)


@pytest.mark.parametrize("n", [2, 11, 2000, 10000, 10001, 60000, 200000, 1_000_000, 4_000_000, 2**31 + 5])
def test_library_pair_counts_equal_the_oracle_at_every_size(lib, orc, n):
    # decide_num_pairs (lib.rs:565-597) as the library computes it in f32, read back through the C ABI
    # (pacmap_generate_pairs with no output buffers needs no device), against the oracle's restatement
    for cfg_kw, orc_kw in [({}, {}), ({"mid_near_ratio": 0.3, "far_pair_ratio": 1.5}, {"mn_ratio": 0.3, "fp_ratio": 1.5}),
                           ({"override_neighbors": 7}, {"override": 7})]:
        got = lib.decide_num_pairs(n, lib.Configuration(**cfg_kw))
        rc, (k, n_mn, n_fp) = orc.decide_num_pairs(n, **orc_kw)
        assert rc == 0
        assert got == (min(k, n - 1), n_mn, n_fp), (n, cfg_kw)
    if n in (60000, 200000, 1_000_000, 4_000_000):
        assert lib.decide_num_pairs(n) == {60000: (22, 11, 44), 200000: (30, 15, 60), 1_000_000: (40, 20, 80),
                                          4_000_000: (49, 25, 98)}[n]
