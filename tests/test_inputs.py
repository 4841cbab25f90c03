"""ParmParse-format input decks (electrostatic_b200.inputs), host only.

The deck below is written for these tests in the reference's format: constants
through my_constants, expressions with functions, NS_default / CNT_default
layers under the structure's own keys, a later line overriding an earlier
one, quoted tokens and comments.  The descriptor built from it must give the
same energy grids as the oracle built from the expected parameters.
"""
import numpy as np
import pytest

DECK = """
# a biased (19,0) tube
my_constants.m = 19
my_constants.ncells = 3*4 + 2      # 14 unit cells
my_constants.Ef = -0.25
my_constants.bias = 0.3
my_constants.kT_room = 300.
my_constants.width = sqrt(4.0)*2   # 4

transport.NS_names = tubeA tubeB
transport.Broyden_fraction = 0.2
transport.Broyden_max_norm = 1.e-6
transport.Broyden_norm_type = absolute
transport.reset_with_previous_charge_distribution = 1

NS_default.contact_T = kT_room kT_room
NS_default.eq_integration_pts = 20 20 40
NS_default.E_valence_min = -8
NS_default.num_modes = 2
CNT_default.gamma = 2.7
CNT_default.type_id = 17 0

tubeA.type = CNT
tubeA.type_id = m 0          # overrides CNT_default
tubeA.num_unitcells = ncells
tubeA.contact_mu_specified = 1
tubeA.contact_mu = Ef Ef-bias
tubeA.num_noneq_paths = 3
tubeA.noneq_integration_pts = 30 width*10 30
tubeA.noneq_percent_intercuts = 25 "50+25"
tubeA.E_zPlus_imag = 1e-3
tubeA.E_pole_max = 2^1 + 1
tubeA.eq_integration_pts = 24 24 48   # the later line wins
tubeA.eq_integration_pts = 16 16 32

tubeB.num_unitcells = 5
tubeB.contact_Fermi_level = Ef
"""


def test_deck_values_and_layers():
    from electrostatic_b200.inputs import Deck
    d = Deck(DECK)
    tr = d.transport()
    assert tr["NS_names"] == ["tubeA", "tubeB"]
    assert tr["Broyden_fraction"] == 0.2 and tr["Broyden_max_norm"] == 1e-6
    assert tr["Broyden_norm_type"] == "absolute" and tr["reset_with_previous_charge_distribution"] == 1
    assert tr["Broyden_threshold_maxstep"] == 200  # the reference's default
    a = d.tube_kwargs("tubeA")
    assert a["type_id"] == (19, 0) and a["num_unitcells"] == 14 and a["gamma"] == 2.7
    assert a["contact_mu"] == (-0.25, -0.55) and a["contact_T"] == (300.0, 300.0)
    assert a["eq_integration_pts"] == (16, 16, 32) and a["noneq_integration_pts"] == (30, 40, 30)
    assert a["noneq_percent_intercuts"] == (25.0, 75.0) and a["E_pole_max"] == 3.0
    assert a["num_modes"] == 2 and a["E_valence_min"] == -8.0
    b = d.tube_kwargs("tubeB", num_modes=3)
    assert b["type_id"] == (17, 0) and b["contact_mu"] == (-0.25, -0.25) and b["num_modes"] == 3


def test_deck_errors():
    from electrostatic_b200.inputs import Deck, DeckError
    with pytest.raises(DeckError, match="unknown symbol"):
        Deck("x.a = nothere + 1").query("x", "a")
    with pytest.raises(DeckError, match="refers to itself"):
        Deck("my_constants.a = a + 1\nx.b = a").query("x", "b")
    with pytest.raises(DeckError, match="integer"):
        Deck("x.n = 2.5").query("x", "n", kind=int)
    with pytest.raises(DeckError, match="needs 2 values"):
        Deck("x.mu = 0.1").query_arr("x", "mu", 2)
    with pytest.raises(DeckError, match="expected 'key = value'"):
        Deck("just words")
    with pytest.raises(DeckError, match="unsupported"):
        Deck("x.a = __import__('os')").query("x", "a")


def test_deck_descriptor_grids_match_oracle(oracle):
    from electrostatic_b200.inputs import Deck
    from electrostatic_b200.negf import desc_energy_points, tube_desc
    kw = Deck(DECK).tube_kwargs("tubeA")
    desc = tube_desc(**kw)
    o = oracle.OracleTube(**{k: v for k, v in kw.items() if k != "precision"})
    for kind in (0, 1, 3):
        E, w, J = desc_energy_points(desc, kind)
        Eo, wo, Jo = o.paths(kind)
        assert len(E) == len(Eo) > 0
        np.testing.assert_allclose(E, Eo, rtol=0, atol=1e-12)
        np.testing.assert_allclose(w * J, wo * Jo, rtol=1e-12, atol=1e-15)
