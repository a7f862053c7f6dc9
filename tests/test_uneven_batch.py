"""Frame specs of the uneven-batch workload (experiments/uneven_batch.py):
seeded, 3:2, multiples of the X-Trans period, within 12-45 MP (rounded down to
the period) and 8256x5504, Bayer sizes accepted by AMaZE's tiling."""
import imops_b200 as im
from experiments.uneven_batch import MAX_H, MAX_W, PERIOD, frame_spec


def test_frame_specs():
    specs = [frame_spec(i, im.amaze_size_supported) for i in range(16)]
    assert specs == [frame_spec(i, im.amaze_size_supported) for i in range(16)]
    assert [s["seed"] for s in specs] == list(range(1000, 1016))
    assert {s["sensor"] for s in specs} == {"bayer", "xtrans"}
    for s in specs:
        W, H = s["W"], s["H"]
        assert W % PERIOD == 0 and H % PERIOD == 0
        assert W <= MAX_W and H <= MAX_H
        assert abs(W / H - 1.5) < 0.01
        assert 11.9e6 <= W * H <= 45e6
        if s["sensor"] == "bayer":
            assert im.amaze_size_supported(W, H)


def test_balanced_bins_split_the_batch():
    """Size-balanced bins over ranks: every frame in exactly one bin, the same
    split on every rank, and the largest bin within one frame of the mean
    load (the greedy bound)."""
    from experiments.uneven_batch import balanced_bins, frame_cost
    specs = [frame_spec(i, im.amaze_size_supported) for i in range(16)]
    for world in (1, 2, 3, 4, 8):
        bins = balanced_bins(specs, world)
        assert bins == balanced_bins(specs, world)
        assert sorted(i for b in bins for i in b) == list(range(16))
        loads = [sum(frame_cost(specs[i]) for i in b) for b in bins]
        assert max(loads) <= sum(loads) / world + max(frame_cost(s) for s in specs)
    assert balanced_bins(specs, 1) == [list(range(16))]
