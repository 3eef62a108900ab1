"""The figures ``bench.py`` divides by (no GPU): algorithmic bytes per node and
system of every launch of one BiCGSTAB iteration, and the DRAM traffic lines
it reads from the committed ncu summaries."""
import bench


def test_iteration_bytes():
    # fixed preconditioner: r,v,t,p,y -> r,p,y,w; two transforms of w per
    # half; the two stencil halves; the residual pass idle in fresh batches
    assert list(bench.KERNEL_BYTES) == ["fwd_h0", "cols_h0", "rinv_h0", "inv_h0", "fwd_h1", "cols_h1", "rinv_h1",
                                        "res_h1", "inv_h1"]
    assert sum(bench.KERNEL_BYTES.values()) == 224
    # learned: inner gain (fwd), multiplier plane (cols), outer gain (rinv)
    extra = {k: bench.LEARNED_BYTES[k] - bench.KERNEL_BYTES[k] for k in bench.KERNEL_BYTES}
    assert extra == {"fwd_h0": 8, "cols_h0": 8, "rinv_h0": 8, "inv_h0": 0, "fwd_h1": 8, "cols_h1": 8, "rinv_h1": 8,
                     "res_h1": 0, "inv_h1": 0}
    assert sum(bench.LEARNED_BYTES.values()) == 272
    assert set(bench.COEF_BYTES) == {"inv_h0", "inv_h1"}


def test_profiled_traffic_of_both_arms():
    # the dominant launches of both arms have a measured traffic line, and it
    # is of the order of their algorithmic bytes (re-reads would show above)
    for arm, table in (("learned", bench.LEARNED_BYTES), ("plain", bench.KERNEL_BYTES)):
        for kernel in ("fwd_h0", "inv_h1"):
            t = bench.profiled_traffic(arm, kernel)
            assert t is not None, (arm, kernel)
            assert 0.5 * table[kernel] < t < 1.2 * (table[kernel] + bench.COEF_BYTES.get(kernel, 0)), (arm, kernel, t)
    assert bench.profiled_traffic("learned", "no_such_kernel") is None
