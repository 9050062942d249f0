"""The HDF5 self-energy cache against the reference's format, on the CPU.

``tests/golden/hdf5_keys.npz`` holds the group / dataset names the reference's
``write_to_hdf5`` (negf/lead_property.py:932-941) creates for a k grid and an
energy grid, with the data it stores.  Through the dict-backed h5py stand-in
(tests/fake_h5py.py; h5py is not installed here):
  * ``compute_all_self_energy`` writes exactly those names and values, so the
    reference's ``read_from_hdf5`` (:944-951), which looks up the names its
    writer makes, reads a cache written here;
  * a file laid out as the reference writes it is read back here by
    ``LeadProperty._load_self_energy`` (the ``use_saved_se`` path).
"""
import sys

import numpy as np
import pytest
import torch

from tests import fake_h5py
from tests.goldens import Golden


@pytest.fixture()
def h5(monkeypatch):
    fake_h5py.FILES.clear()
    monkeypatch.setitem(sys.modules, "h5py", fake_h5py.module())
    yield fake_h5py
    fake_h5py.FILES.clear()


class _Lead:
    """What compute_all_self_energy needs of a LeadProperty: tab, results_path, self_energy_cal."""

    def __init__(self, tab, g, kgrid):
        self.tab = tab
        self.results_path = "/fake-results"
        self._g, self._kgrid = g, kgrid

    def self_energy_cal(self, kpoint, energy, eta_lead=1e-5, **kw):
        ik = int(np.argmin(np.abs(self._kgrid - np.asarray(kpoint, dtype=float)).sum(-1)))
        side = "L" if self.tab == "lead_L" else "R"
        n_e = int(np.asarray(energy).reshape(-1).shape[0])
        return torch.stack([torch.as_tensor(self._g[f"se/{side}/{ik}/{ie}"]) for ie in range(n_e)])


def _names(path, tab):
    return sorted(f"{tab}|{g}|{d}" for g, ds in fake_h5py.keys(path).items() for d in ds)


def test_cache_written_here_has_the_reference_layout(h5, tmp_path):
    from dpnegf_b200.lead_property import compute_all_self_energy
    g = Golden("hdf5_keys")
    kgrid, egrid = g["kgrid"], g["egrid"]
    leads = [_Lead("lead_L", g, kgrid), _Lead("lead_R", g, kgrid)]
    out = compute_all_self_energy(1e-5, leads[0], leads[1], kgrid, egrid, self_energy_save_path=str(tmp_path),
                                  save_format="h5")
    names = _names(tmp_path / "self_energy_leadL.h5", "L") + _names(tmp_path / "self_energy_leadR.h5", "R")
    assert sorted(names) == sorted(str(x) for x in g["names"])
    for tab, side in (("lead_L", "L"), ("lead_R", "R")):
        stored = fake_h5py.keys(tmp_path / f"self_energy_lead{side}.h5")
        for ik, k in enumerate(kgrid):
            for ie, e in enumerate(egrid):
                grp, ds = f"E_{e:.8f}", f"k_{k[0]}_{k[1]}_{k[2]}"
                assert np.array_equal(stored[grp][ds], g[f"se/{side}/{ik}/{ie}"])
            key = tuple(float(x) for x in k)
            assert torch.equal(out[tab][key][2], torch.as_tensor(g[f"se/{side}/{ik}/2"]))


def test_cache_in_the_reference_layout_is_read_here(h5):
    from dpnegf_b200.lead_property import LeadProperty
    g = Golden("hdf5_keys")
    kgrid, egrid = g["kgrid"], g["egrid"]
    # lay the file out from the recorded names alone, as the reference's writer left it
    for name in g["names"]:
        side, grp, ds = str(name).split("|")
        ik = next(i for i, k in enumerate(kgrid) if ds == f"k_{k[0]}_{k[1]}_{k[2]}")
        ie = next(i for i, e in enumerate(egrid) if grp == f"E_{e:.8f}")
        with fake_h5py.File(f"/ref/self_energy_lead{side}.h5", "a") as f:
            f.require_group(grp).create_dataset(ds, data=g[f"se/{side}/{ik}/{ie}"], compression="gzip")
    for side in ("L", "R"):
        for ik, k in enumerate(kgrid):
            for ie, e in enumerate(egrid):
                se = LeadProperty._load_self_energy(f"/ref/self_energy_lead{side}.h5", k,
                                                    torch.tensor(e, dtype=torch.float64), "h5")
                assert se.dtype == torch.complex128
                assert np.array_equal(se.numpy(), g[f"se/{side}/{ik}/{ie}"])
    with pytest.raises(KeyError):
        LeadProperty._load_self_energy("/ref/self_energy_leadL.h5", kgrid[0], torch.tensor(0.777), "h5")
