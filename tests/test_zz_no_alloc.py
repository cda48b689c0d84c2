"""htf_projection_noalloc: the projector on caller-owned device vectors,
with no allocation.  Callers that cannot allocate while they project — a
serving loop held to a fixed device-memory budget, a latency-bound loop that
must not trigger the synchronisation an allocation can cause — use it; its
reduction scratch is a static device array shared by all calls.  Checked
against the existing htf_projection (host buffers) on two calls in a row,
with the projector tolerance of the other GPU tests (1e-12 relative), and a
host pointer is refused with HTF_EINVAL before anything is launched.
Collected last on purpose."""
import numpy as np
import pytest

import hfls_b200 as hb

pytestmark = pytest.mark.gpu


def test_projection_noalloc_matches_projection_twice():
    import torch

    spec = hb.mesh_spec(clusters=(2, 1, 1), subs=(2, 2, 2), elems=(3, 3, 3), jitter=0.1, seed=4,
                        material=hb.HTF_MAT_LOGUNIFORM, E=1.0, E_hi=1e3)
    m = hb.generate_mesh(spec)
    s = hb.Solver({"typeBc": "cor", "preconditioner": "Dirichlet_explicit", "device": "0"})
    s.set_mesh(m)
    s.setup()
    n = s.n_lambda()
    rng = np.random.default_rng(11)
    stream = torch.cuda.current_stream()
    for _ in range(2):
        x = rng.standard_normal(n)
        ref = s.projection(x[None])[0]
        xd = torch.from_numpy(x).to("cuda:0")
        pd = torch.full_like(xd, float("nan"))
        s.projection_noalloc(xd.data_ptr(), pd.data_ptr(), stream.cuda_stream)
        stream.synchronize()
        got = pd.cpu().numpy()
        assert np.all(np.isfinite(got))
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-12


def test_projection_noalloc_refuses_host_memory():
    spec = hb.mesh_spec(clusters=(1, 1, 1), subs=(2, 1, 1), elems=(2, 2, 2))
    s = hb.Solver({"typeBc": "cor", "device": "0"})
    s.set_mesh(hb.generate_mesh(spec))
    s.setup()
    x = np.ones(s.n_lambda())
    y = np.zeros_like(x)
    with pytest.raises(hb.HTFError) as e:
        s.projection_noalloc(x.ctypes.data, y.ctypes.data, 0)
    assert e.value.code == hb.HTF_EINVAL
