"""GPU parity against the reference's own CPU code, run here rather than
through golden vectors: seeded workloads of every configuration's shape,
verified on the GPU through the C ABI and by the reference's
computeAllQueriesCPU (src-integration/myers-reorderBuffer-padding.c:178-208,
aligned windows) and its exact-window Myers (src/myers-4bits.c:75-153),
both compiled from the reference's sources into oracle/_ref/. Integer
outputs: bit-exact. Skipped when oracle/_ref/ was not built (the reference
checkout was absent at build time)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DIST = 0.2
REF_SIZE = 8_000_000


@pytest.fixture(scope="module")
def gpu(mg, orc, cuda_ok):
    if not orc.have_reference():
        pytest.skip("oracle/_ref/ not built")
    import torch
    torch.cuda.init()
    return mg


@pytest.fixture(scope="module")
def data(gpu):
    ref_words = gpu.make_reference(REF_SIZE, 2468)
    ref = gpu.Reference(ref_words, REF_SIZE)
    yield ref_words, ref
    ref.close()


def _gpu_results(mg, ref, w, window, path, min_size=0, max_size=0):
    ctx = mg.Context(len(w["cands"]))
    try:
        return mg.verify_torch(ctx, ref, w["peq"], w["qinfo"], w["cands"], DIST, window=window, path=path,
                               min_size=min_size, max_size=max_size)
    finally:
        ctx.close()


# workload -> scale: about 10K-60K candidates each (the long reads' CPU time bounds theirs)
SCALES = {1: 0.05, 2: 0.005, 3: 0.002, 4: 0.01}


@pytest.mark.parametrize("k", sorted(SCALES))
@pytest.mark.parametrize("path", ["plain", "batched"])
def test_aligned_vs_reference(gpu, orc, data, k, path):
    ref_words, ref = data
    w = gpu.make_workload(gpu.workload_spec(k, scale=SCALES[k], ref_size=REF_SIZE), ref_words)
    expect, _ = orc.reference_verify_aligned(w["peq"], w["qinfo"], w["cands"], ref_words, REF_SIZE, DIST,
                                             uncapped=True)
    got = _gpu_results(gpu, ref, w, gpu.WINDOW_ALIGNED, gpu.PATH_PLAIN if path == "plain" else gpu.PATH_BATCHED)
    bad = np.nonzero(got != expect)[0]
    assert bad.size == 0, (k, path, len(bad), got[bad[:5]], expect[bad[:5]])


@pytest.mark.parametrize("k", [1, 2])
@pytest.mark.parametrize("path", ["plain", "batched"])
def test_exact_vs_reference(gpu, orc, data, k, path):
    """The reference's exact-window Myers takes one query length per run:
    the fixed-length workloads (100 and 1,000 bases)."""
    ref_words, ref = data
    w = gpu.make_workload(gpu.workload_spec(k, scale=SCALES[k], ref_size=REF_SIZE), ref_words)
    m = int(w["qinfo"]["size"][0])
    assert (w["qinfo"]["size"] == m).all()
    expect, _ = orc.reference_verify_exact(w["peq"], w["qinfo"], w["cands"], ref_words, REF_SIZE, DIST)
    got = _gpu_results(gpu, ref, w, gpu.WINDOW_EXACT, gpu.PATH_PLAIN if path == "plain" else gpu.PATH_BATCHED,
                       m, m)
    bad = np.nonzero(got != expect)[0]
    assert bad.size == 0, (k, path, len(bad), got[bad[:5]], expect[bad[:5]])
