"""Batched simulations on separate streams with CUDA-graph chunks give the
same states as the same simulations stepped one at a time."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_graph_chunks_match_sequential(fundem):
    from fundem_b200 import batch
    scs, params = batch.calibration_scenarios(n_sims=6, seed=3, n_min=200, n_max=1500)
    a = batch.Batch(scs)
    b = batch.Batch(scs)
    a.run_graphs(60, 25)          # chunks of 25, 25, 10: two graphs recorded
    b.run_sequential(60)
    for sa, sb in zip(a.sims, b.sims):
        xa, xb = sa.state(), sb.state()
        assert np.array_equal(xa["pos"], xb["pos"]) and np.array_equal(xa["vel"], xb["vel"])
    best, times = batch.autotune_chunk(a, candidates=(10, 30), probe_steps=30)
    assert best in (10, 30) and all(t > 0 for t in times.values())
    a.close()
    b.close()


def test_step_graph_matches_step(fundem):
    from fundem_b200 import workloads
    sim, sc, info = workloads.bonded_column(n=2048, footprint=(16, 16), seed=2, settle_steps=0)
    sim.close()
    import torch
    st = torch.cuda.Stream()
    g = fundem.Simulation.from_scenario(sc, records=False, stream=st.cuda_stream)
    p = fundem.Simulation.from_scenario(sc, records=False)
    g.detect(); p.detect()
    for _ in range(3):
        g.step_graph(20)
    p.step(60)
    g.sync(); p.sync()
    assert np.array_equal(g.state()["pos"], p.state()["pos"])
    assert g.num_contacts(fundem.PP) == p.num_contacts(fundem.PP)
    g.close(); p.close()


@pytest.mark.parametrize("chunks", [(1,) * 12, (3, 1, 3, 5), (2, 1, 1, 8)])
def test_step_graph_odd_lengths_and_mixed_calls(fundem, chunks):
    """Graphs of odd length alternate the contact-list generation they start
    on, and plain steps may come between replays: every sequence equals the
    same number of plain steps bit for bit."""
    from fundem_b200 import workloads
    sim, sc, info = workloads.bonded_column(n=2048, footprint=(16, 16), seed=2, settle_steps=0)
    sim.close()
    g = fundem.Simulation.from_scenario(sc, records=False)
    p = fundem.Simulation.from_scenario(sc, records=False)
    g.detect(); p.detect()
    total = 0
    for i, c in enumerate(chunks):
        g.step_graph(c)
        if i % 2 == 1:
            g.step(1)  # a plain step between replays flips the generation too
            total += 1
        total += c
    p.step(total)
    g.sync(); p.sync()
    assert np.array_equal(g.state()["pos"], p.state()["pos"])
    for k in (fundem.PP, fundem.PW):
        assert g.num_contacts(k) == p.num_contacts(k)
    g.close(); p.close()
