"""Recovery driver host logic: YAML flattening, type coercion and enum checks
(Recovery.py:44-72)."""
import importlib

import pytest

from conftest import PKG_NAME


def rec():
    return importlib.import_module(PKG_NAME + ".recovery")


def test_load_config_flattens_and_coerces(tmp_path):
    p = tmp_path / "c.yaml"
    p.write_text("data:\n  data_dir: d\n  gap: '2'\nphysics:\n  wavelength: 2.4e-9\nmodel:\n"
                 "  n_levels: 16\n  per_level_scale: '1.5'\n  init_type: initProbe\ntraining:\n"
                 "  iters: '10'\n  lr: '1e-3'\n  loss_type: Poisson_likelihood_loss\n")
    cfg = rec().load_config(str(p))
    assert cfg["data_dir"] == "d" and cfg["gap"] == 2 and cfg["iters"] == 10
    assert isinstance(cfg["lr"], float) and cfg["lr"] == 1e-3
    assert isinstance(cfg["per_level_scale"], float) and cfg["wavelength"] == 2.4e-9
    assert cfg["loss_type"] == "Poisson_likelihood_loss"


@pytest.mark.parametrize("key,val", [("init_type", "initFoo"), ("loss_type", "L2"), ("model_type", "mlp")])
def test_load_config_rejects_bad_enums(tmp_path, key, val):
    p = tmp_path / "c.yaml"
    p.write_text(f"model:\n  {key}: {val}\n")
    with pytest.raises(ValueError):
        rec().load_config(str(p))


def test_reference_configs_parse():
    import os
    import glob
    from conftest import ROOT
    ref = os.path.join(os.environ.get("PTYCHO_REFERENCE", "/root/reference"), "config")
    if not os.path.isdir(ref):
        pytest.skip("reference tree not present")
    for f in glob.glob(os.path.join(ref, "*.yaml")):
        cfg = rec().load_config(f)
        assert cfg["loss_type"] in rec().VALID_LOSS_TYPES
