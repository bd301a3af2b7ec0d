"""The learned model file (pacmap_model_save / pacmap_model_load: checksummed, shape-checked) and the
target standardisation, on the host -- no GPU is needed for either."""
import numpy as np
import pytest


def _model(lib, d=24, dim=3, seed=0):
    L = lib.learned
    rng = np.random.default_rng(seed)
    return L.LearnedModel(params=rng.normal(size=L.param_count(d, dim)).astype(np.float32), d=d, dim=dim,
                          pre_min=-3.25, pre_max=7.5, pre_mean=rng.normal(size=d).astype(np.float32),
                          target_mean=rng.normal(size=dim).astype(np.float32),
                          target_std=rng.uniform(0.5, 4.0, size=dim).astype(np.float32))


def _same(a, b):
    assert a.d == b.d and a.dim == b.dim
    assert np.float32(a.pre_min) == np.float32(b.pre_min) and np.float32(a.pre_max) == np.float32(b.pre_max)
    for f in ("params", "pre_mean", "target_mean", "target_std"):
        assert np.array_equal(getattr(a, f), getattr(b, f)), f


@pytest.mark.parametrize("d,dim", [(24, 3), (128, 2), (1, 1), (300, 16)])
def test_save_load_round_trip(lib, tmp_path, d, dim):
    m = _model(lib, d, dim, seed=d)
    path = tmp_path / "model.bin"
    m.save(path)
    _same(m, lib.learned.LearnedModel.load(path))
    # header + constants + parameters + checksum, nothing else
    assert path.stat().st_size == 8 + 4 + 4 + 3 * 8 + 4 * (2 + d + 2 * dim + lib.learned.param_count(d, dim)) + 8


def test_damaged_file_is_rejected(lib, tmp_path):
    path = tmp_path / "model.bin"
    _model(lib).save(path)
    raw = bytearray(path.read_bytes())
    for pos in (20, 60, len(raw) // 2, len(raw) - 9, len(raw) - 1):  # header, constants, params, checksum
        bad = bytearray(raw)
        bad[pos] ^= 0x10
        p = tmp_path / f"bad{pos}.bin"
        p.write_bytes(bytes(bad))
        with pytest.raises(lib.ModelFileError):
            lib.learned.LearnedModel.load(p)


def test_truncated_foreign_and_missing_files_are_rejected(lib, tmp_path):
    path = tmp_path / "model.bin"
    _model(lib).save(path)
    raw = path.read_bytes()
    for i, data in enumerate([raw[:-1], raw[: len(raw) // 2], raw[:12], b"", b"not a model at all" * 10]):
        p = tmp_path / f"x{i}.bin"
        p.write_bytes(data)
        with pytest.raises(lib.ModelFileError):
            lib.learned.LearnedModel.load(p)
    with pytest.raises(lib.ModelFileError):
        lib.learned.LearnedModel.load(tmp_path / "does_not_exist.bin")
    with pytest.raises(lib.ModelFileError):
        _model(lib).save(tmp_path / "no_such_dir" / "model.bin")


def test_unsupported_shapes_are_refused(lib, tmp_path):
    m = _model(lib, d=8, dim=2)
    m.dim = 17
    with pytest.raises(lib.Unsupported):
        m.save(tmp_path / "m.bin")


def test_target_stats_is_the_training_standardisation(lib):
    rng = np.random.default_rng(3)
    y = (rng.normal(size=(5000, 3)) * [1e-4, 2.0, 30.0] + [5.0, -1.0, 0.0]).astype(np.float32)
    mean, std = lib.learned.target_stats(y)
    y64 = y.astype(np.float64)
    assert np.allclose(mean, y64.mean(0), rtol=1e-6, atol=0)
    assert np.allclose(std, y64.std(0), rtol=1e-6, atol=0)
    with pytest.raises(lib.EmptyArrayMean):
        lib.learned.target_stats(np.zeros((0, 2), np.float32))
