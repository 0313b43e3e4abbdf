"""Host-side logic of the package checked against the oracle (no GPU)."""
import numpy as np
import pytest

from oracle import phasing_oracle as O


def test_expand_runs_default_and_merge():
    from als_speckle_b200.engine import expand_runs
    assert expand_runs(None) == ([0, 1], [99, 1])
    assert expand_runs((("hio", 5), ("hio", 3), ("er", 2))) == ([0, 1], [8, 2])
    assert expand_runs((("er", 1), ("sf", 2)), quirks="cpu") == ([5, 6], [1, 2])
    with pytest.raises(ValueError):
        expand_runs((("xyz", 3),))
    with pytest.raises(ValueError):
        expand_runs((("hio",),))


def test_order_rotation_matches_cyclic_list():
    from als_speckle_b200.phasing import _runs_from_flat
    from als_speckle_b200.engine import expand_runs
    order = (("hio", 5), ("er", 5), ("sf", 1))
    flat_names = O.expand_order(order)
    algs, counts = expand_runs(order)
    flat = [a for a, c in zip(algs, counts) for _ in range(c)]
    for done in (0, 3, 7, 10, 12):
        rot = [flat[(done + i) % len(flat)] for i in range(len(flat))]
        a2, c2 = expand_runs(_runs_from_flat(rot))
        got = [a for a, c in zip(a2, c2) for _ in range(c)]
        names = {0: "hio", 1: "er", 3: "sf"}
        assert [names[g] for g in got] == [flat_names[(done + i) % len(flat_names)] for i in range(len(flat))]


def test_bounding_box_matches_oracle():
    from als_speckle_b200 import masking
    rng = np.random.default_rng(3)
    for _ in range(50):
        d = np.zeros((40, 40))
        r0, c0 = rng.integers(0, 30, 2)
        d[r0:r0 + rng.integers(1, 10), c0:c0 + rng.integers(1, 10)] = 1
        for pad in (0, 4, 10):
            for sq in (False, True):
                assert tuple(masking.bounding_box(d, pad=pad, force_to_square=sq)) == \
                    tuple(O.bounding_box(d, pad=pad, force_to_square=sq))


def test_label_parts_matches_find_all_objects():
    from als_speckle_b200 import masking
    rng = np.random.default_rng(5)
    for _ in range(20):
        sup = (rng.random((20, 26)) > 0.72).astype(float)
        lab, n = masking.label_parts(sup)
        objs = O.find_all_objects(sup)
        assert n == len(objs)
        for k in range(n):
            assert np.array_equal(lab == k + 1, objs[k].astype(bool))


def test_gaussian_kernel_is_separable_form_of_reference():
    from als_speckle_b200.phasing import _gaussian_1d_kernel
    for shape, s in (((20, 24), 3.0), ((33, 17), 0.7), ((64, 64), 2.0)):
        k2 = np.fft.fftshift(O.gaussian(shape, (s, s)))
        k2 /= k2.sum()
        sep = np.outer(_gaussian_1d_kernel(shape[0], s), _gaussian_1d_kernel(shape[1], s))
        assert np.allclose(sep, k2, rtol=1e-12, atol=1e-300)


def test_synthetic_generator_properties():
    from als_speckle_b200 import synth
    obj, modulus, support = synth.pattern(256, n_ellipses=20, box=64, peak=1e5, seed=1,
                                          support_edge=80)
    assert modulus.shape == (256, 256) and modulus.dtype == np.float32
    assert support.sum() == 80 * 80
    assert abs(float(modulus.max()) ** 2 - 1e5) < 5 * np.sqrt(1e5)  # peak photons, Poisson
    assert np.all(np.abs(obj[np.abs(obj) > 0]) <= 1.0 + 1e-12)
    o2, m2, s2 = synth.pattern(256, n_ellipses=20, box=64, peak=1e5, seed=1, support_edge=80)
    assert np.array_equal(m2, modulus)


def test_tuned_e_table(tmp_path):
    """The engine's default E per size comes from the tuning file's entry for
    the device; sizes without an E and other devices are ignored."""
    import json
    from als_speckle_b200 import autotune
    path = tmp_path / "tune.json"
    path.write_text(json.dumps({
        "Dev A": {"256": {"E": 16, "rate": 1.0}, "512": {"E": 32}, "1024": {"rate": 2.0}},
        "Dev B": {"256": {"E": 32}},
    }))
    assert autotune.tuned_e_per_n(str(path), "Dev A") == {256: 16, 512: 32}
    assert autotune.tuned_e_per_n(str(path), "Dev C") == {}
    assert autotune.tuned_e_per_n(str(tmp_path / "missing.json"), "Dev A") == {}
    # the committed table names E for every size the benchmarks use on B200
    table = autotune.tuned_e_per_n(device_name="NVIDIA B200")
    assert set(table) >= {256, 512, 1024, 2048}
    assert all(e in (8, 16, 32) for e in table.values())


def test_package_exposes_the_modules_example_scripts_use():
    """``import als_speckle_b200 as speckle`` then ``speckle.io.open``,
    ``speckle.phasing.phasing``, ``speckle.phasing.refine_support`` and
    ``speckle.masking.bounding_box``, as the reference's phasing examples
    call them (``examples/basic_phasing_example.py``,
    ``examples/advanced_phasing_example.py``)."""
    import als_speckle_b200 as speckle
    assert callable(speckle.io.open) and callable(speckle.io.save)
    assert callable(speckle.masking.bounding_box)
    for name in ("phasing", "refine_support", "align_global_phase", "prtf", "rftf",
                 "center_of_mass_average", "covar_results", "gpu_prtf", "gpu_rftf"):
        assert callable(getattr(speckle.phasing, name)), name
    for name in ("load", "seed", "iterate", "reconstruct", "optimize_coherence", "status", "get"):
        assert callable(getattr(speckle.phasing.phasing, name)), name
    with pytest.raises(AttributeError):
        speckle.no_such_module
