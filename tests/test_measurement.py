"""The measurement arithmetic of bench.py (no device needed): the
algorithmic bytes of one MD step of the 23,550-atom box with a 64^3 PME grid
(the unique data each phase must move, counted once), the FP32 flops
counted per in-cutoff pair, and the DRAM traffic figures read from the
committed ncu summary."""
import bench


def test_algorithmic_bytes_of_the_benchmark_step():
    ab = bench.algorithmic_bytes_per_step(23550, 64)
    mb = {k: v / 1e6 for k, v in ab.items()}
    # per phase, in MB: pairs 1.60, sort 1.70, spread 2.47, FFTs 6.36,
    # convolution 2.16, gather 3.04, integrator 3.01; 20.3 in all
    want = {"pairs": 1.60, "sort": 1.70, "spread": 2.47, "fft": 6.36, "convolution": 2.16,
            "gather": 3.04, "integrator": 3.01}
    for k, v in want.items():
        assert abs(mb[k] - v) < 0.01, (k, mb[k])
    assert ab["pairs"] == 23550 * 68
    assert ab["total"] == sum(v for k, v in ab.items() if k != "total") == 20344184


def test_pair_flop_count():
    """FMA counts two: difference 3, r^2 5, charge product 1, 1/r^2 1, r^-6 2,
    B r^-6 1, A r^-12 2, LJ force 4, C2 switch 15, Ewald table cubic 8 and
    charge 1, pair forces on i and j 12."""
    items = [3, 5, 1, 1, 2, 1, 2, 4, 15, 8, 1, 12]
    assert bench.PAIR_FLOPS == sum(items) == 55


def test_traffic_figures():
    cold, warm = bench.load_traffic()
    pair_bytes = bench.algorithmic_bytes_per_step(23550, 64)["pairs"]
    # cold caches: the list (about 10.7 MB of j-lane entries) is read from
    # DRAM; in the MD loop it stays in L2
    assert cold > pair_bytes > warm > 0
