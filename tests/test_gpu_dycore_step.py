"""One time step's transforms of the primitive-equation wet model (T63, 8 layers), in the
reference's order (SpeedyWeather/src/time_stepping/transform.jl:117-191,
SpeedyWeather/src/dynamics/tendencies.jl:161-214): captured as one CUDA graph and
replayed, the results equal the eager calls bit for bit."""
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp32", "bf16x3"])
def test_graph_replay_equals_eager(precision):
    import torch
    import speedytransforms as st
    step = st.DycoreStep(T=63, nlat_half=48, L=8, precision=precision)
    outs = lambda: [step.grid_prog.data, step.uv_grid.data, step.dpres_grid.data, step.spec_tend.data,  # noqa: E731
                    step.tend.data]
    step()
    torch.cuda.synchronize()
    eager = [o.clone() for o in outs()]
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        step()
    torch.cuda.current_stream().wait_stream(side)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        step()
    for o in outs():
        o.zero_()
    graph.replay()
    torch.cuda.synchronize()
    for a, b in zip(outs(), eager):
        assert torch.equal(a, b)
    graph.replay()                          # replays again (the step resets its accumulators)
    torch.cuda.synchronize()
    for a, b in zip(outs(), eager):
        assert torch.equal(a, b)
    assert step.S.device_status() == 0
