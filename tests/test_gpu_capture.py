"""A caller's own CUDA graph can hold the cycle: lulesh_step on a stream
that the caller is capturing enqueues the cycle's kernels into that graph.
Replaying it equals stepping the set directly, bit for bit."""
import pytest

pytestmark = pytest.mark.gpu


def _capture(torch, s, stream, n):
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=stream):
        s.step(n)
    return g


@pytest.mark.parametrize("kind", ["single", "subdomains", "batch"])
def test_replayed_capture_equals_direct_steps(lulesh, kind):
    torch = pytest.importorskip("torch")
    stream = torch.cuda.Stream()

    def make():
        if kind == "single":
            return lulesh.LuleshSet(nx=20, its=-1)
        if kind == "subdomains":
            return lulesh.LuleshSet(nx=6, tp=2, its=-1, flags=lulesh.FLAG_COMM_STAGED)
        return lulesh.LuleshSet.batch([lulesh.JobSpec(9, its=-1), lulesh.JobSpec(14, its=-1)])

    with make() as a, make() as b:
        a.set_stream(stream.cuda_stream)
        a.step(0)  # prepares the set outside the capture
        g = _capture(torch, a, stream, 7)
        for _ in range(3):
            g.replay()
        torch.cuda.synchronize()
        b.step(21)
        b.sync()
        for j in range(2 if kind == "batch" else 1):
            assert a.state(j) == b.state(j)
        assert a.state()["cycle"] == 21
        for f in ("e", "x", "xd"):
            assert (a.field(f) == b.field(f)).all(), f
        del g


def test_capture_needs_a_prepared_set(lulesh):
    torch = pytest.importorskip("torch")
    stream = torch.cuda.Stream()
    with lulesh.LuleshSet(nx=8, its=-1) as s:
        s.set_stream(stream.cuda_stream)
        g = torch.cuda.CUDAGraph()
        with pytest.raises(lulesh.LuleshError) as ei:
            with torch.cuda.graph(g, stream=stream):
                s.step(1)
        assert ei.value.status == lulesh.INVALID_ARG
