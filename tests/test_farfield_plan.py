"""The far field's choice between one sum per direction and one z sum per distinct kz
(plan_kz_groups through ddagpu_farfield_plan, host code; no device needed)."""
import numpy as np
import pytest

import dda_fft_b200 as D


def test_fixed_orientation_planes_share_kz(oracle):
    """12 planes about the incident direction (main.cpp:376-387): 181 angles, 181 groups;
    the pair of polarisations shares them; the mid configuration's sphere takes the grouped
    form."""
    _, ksc = oracle.scattering_geometry(12, 181, 0.0, 1.0)
    assert D.farfield_plan(ksc, 64, 137376) == (181, 181)
    pair = np.stack([ksc, ksc])
    assert D.farfield_plan(pair, 64, 137376, nrhs=2, pairs=True) == (181, 181)
    # without pairing each right-hand side is a block of its own: the same groups
    assert D.farfield_plan(pair, 64, 137376, nrhs=2) == (181, 181)


def test_distinct_kz_keeps_the_direct_sum(oracle):
    """One plane of 19 angles: every direction its own kz, so grouping saves nothing and
    the default keeps the per-direction sum; mode 2 groups anyway, mode 1 never."""
    _, ksc = oracle.scattering_geometry(1, 19, 0.0, 10.0)
    assert D.farfield_plan(ksc, 32, 17000) == (0, 0)
    assert D.farfield_plan(ksc, 32, 17000, mode=2) == (19, 19)
    _, many = oracle.scattering_geometry(12, 181, 0.0, 1.0)
    assert D.farfield_plan(many, 64, 137376, mode=1) == (0, 0)


def test_rotated_orientations_stay_direct(oracle):
    """Monte-Carlo orientations rotate the planes off the lattice axes: kz no longer repeats."""
    _, ksc = oracle.scattering_geometry(12, 181, 0.0, 1.0)
    rot = D.mc_rotations(7, 2)
    ks = np.stack([ksc.reshape(-1, 3) @ r.T for r in rot])
    g, _ = D.farfield_plan(ks, 64, 137376, nrhs=2)
    assert g == 0


def test_items_split_large_groups_and_sparse_targets(oracle):
    """A group of more than 16 directions takes several work items; a sparse target (few
    active cells) keeps the direct sum, which only visits active cells."""
    _, ksc = oracle.scattering_geometry(40, 7, 0.0, 30.0)    # 7 groups of 40 directions
    g, items = D.farfield_plan(ksc, 64, 137376)
    assert g == 7 and items == 7 * 3
    assert D.farfield_plan(ksc, 64, 500) == (0, 0)


def test_non_finite_directions_and_bad_arguments():
    ks = np.zeros((10, 3))
    ks[:, 2] = 1.0
    ks[3, 0] = np.nan
    assert D.farfield_plan(ks, 16, 4096, mode=2) == (0, 0)
    with pytest.raises(D.DDAGPUError):
        D.farfield_plan(np.ones((4, 3)), 16, 100, mode=3)
    with pytest.raises(D.DDAGPUError):
        D.farfield_plan(np.ones((4, 3)), (16, 0, 16), 100)
