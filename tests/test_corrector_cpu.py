"""Corrector host logic without a GPU: architecture size, initialisation, the
CPU oracle network's shapes and the dataset configuration pairing."""
import torch

from aeromhd_cuda_b200.corrector import architecture, init_params, n_params
from aeromhd_cuda_b200.learned import T_SNAPS, paired_configs


def test_architecture_is_a_4_level_32_to_256_unet_of_about_0p6M_params():
    specs = architecture()
    assert [s.cout for s in specs if s.name.startswith("e")] == [32, 64, 128, 256]
    assert all(s.k in (1, 3) for s in specs) and specs[-1].cout == 10 and specs[0].cin == 10
    n = n_params(specs)
    assert 550_000 < n < 700_000, n


def test_oracle_network_runs_and_matches_parameter_count():
    import nn_oracle
    specs = architecture()
    p = init_params(specs, seed=1)
    assert sum(v["w"].numel() + v["b"].numel() for v in p.values()) == n_params(specs)
    y = nn_oracle.forward(p, torch.randn(2, 10, 32, 16))
    assert y.shape == (2, 10, 32, 16)
    a = torch.randn(10, 2 * 32 * 16)
    assert torch.equal(nn_oracle.from_nchw(nn_oracle.to_nchw(a, 2, 32, 16)), a)


def test_init_is_seeded():
    a, b = init_params(architecture(), 3), init_params(architecture(), 3)
    assert all(torch.equal(a[k]["w"], b[k]["w"]) for k in a)
    assert not torch.equal(init_params(architecture(), 4)["e1"]["w"], a["e1"]["w"])


def test_pairs_share_parameters_and_differ_by_4x_resolution():
    c, f = paired_configs([1, 2, 3], nyc=64)
    for a, b in zip(c, f):
        assert (b.nx, b.ny) == (4 * a.nx, 4 * a.ny) and (a.nx, a.ny) == (256, 64)
        assert (a.mach, a.density_ratio, a.bx0, a.b1, a.perturbation_mode) == \
               (b.mach, b.density_ratio, b.bx0, b.b1, b.perturbation_mode)
        assert a.ic_frame == "post_shock" and a.noise_amp == 0.0
    assert len(T_SNAPS) == 30 and abs(T_SNAPS[-1] - 3.0) < 1e-12


def test_linear_prolongation_keeps_every_coarse_mean():
    """prolong_linear: 4x4 sub-cells whose average is the coarse cell, exact on a
    linear field away from the limited x ends."""
    from aeromhd_cuda_b200.learned import prolong_linear
    g = torch.Generator().manual_seed(3)
    U = torch.randn(10, 12, 8, generator=g, dtype=torch.float64)
    F = prolong_linear(U, 4)
    assert F.shape == (10, 48, 32)
    assert torch.allclose(F.reshape(10, 12, 4, 8, 4).mean(dim=(2, 4)), U, atol=1e-13)
    x = torch.arange(12, dtype=torch.float64)[:, None].expand(12, 8)
    lin = prolong_linear(x.expand(10, 12, 8).clone(), 4)
    fine_x = (torch.arange(48, dtype=torch.float64) + 0.5) / 4 - 0.5
    assert torch.allclose(lin[0, 4:-4, 0], fine_x[4:-4])
