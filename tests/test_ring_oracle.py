"""The ring-slot oracle (oracle/ring.py) against the reference's own
schreibe_slot (film_producer.py:87-123) and the self-gravity row reorder of
its producer loop (:1245-1261), written by tests/golden/make_golden.py."""
import numpy as np
import pytest

from oracle import ring as orng


@pytest.mark.parametrize("case", ["none", "few", "overflow"])
def test_slot_bytes_match_reference(load_golden, case):
    g = load_golden("ring_slots.npz")
    n, m_sub = int(g["n"]), int(g["m_sub"])
    sub_max = int(g[f"{case}_sub_max"])
    sub_i = None if case == "none" else (g[f"{case}_idx"], g[f"{case}_pos"])
    slot, over = orng.write_slot(n, m_sub, sub_max, g["out_i"], sub_i)
    assert len(slot) == orng.slot_bytes(n, m_sub, sub_max)
    assert np.array_equal(np.frombuffer(slot, np.uint8), g[f"{case}_slot"])
    assert over == bool(g[f"{case}_overflow"])


def test_selfgrav_reorder_matches_reference(load_golden):
    g = load_golden("ring_slots.npz")
    full = orng.reorder_selfgrav(g["sg_outs"], g["sg_m"], g["sg_t"], int(g["sg_n"]))
    assert np.array_equal(full, g["sg_full"])
