"""Host side of the ensemble: the seeded parameter set of the batched benchmark."""
from vlasov1d2v_b200.ensemble import sample_members


def test_sample_members_is_seeded_and_bounded():
    a = sample_members(64, seed=0)
    b = sample_members(64, seed=0)
    assert a == b and len(a) == 64
    for q in a:
        nx, nu, nv = q["res"]
        assert nx in (8, 16, 32) and nu == nv and nu in (24, 32, 40) and q["order"] in (6, 7, 8, 9)
        assert nx * nu * nv * q["order"] ** 3 <= 2.4e6
        assert 0.5 <= q["k"] <= 2.0 and q["ring_j"] in (3, 4, 5, 6) and 5 <= q["om_pc"] <= 15
        assert 1e-4 <= q["amp"] <= 1e-2
    assert len({(q["res"], q["order"]) for q in a}) >= 4   # heterogeneous grids and orders
