"""GPU modelling engine (b200_batch_*): forward traces and adjoint gradients of batched shots
against the FP64 oracle (oracle/oracle_model.c), checkpoint and batch invariance, CUDA graphs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ORDER, DX, NT, F0 = 8, 10.0, 150, 30.0


@pytest.fixture(scope="module")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hpcscan_b200.grid import init_device
    init_device(0)
    return torch


def make_shots(torch, sizes=((36, 30, 40), (28, 36, 24)), seed=0, scale=1.0, dobs=None):
    from hpcscan_b200.modeling import Shot, grf_velocity
    shots = []
    for i, n in enumerate(sizes):
        vel = grf_velocity((n[2], n[1], n[0]), sigma=3.0, seed=seed + i, vmin=1600.0, vmax=2600.0)
        if scale != 1.0:
            z, y, x = torch.meshgrid(*[torch.arange(k, device=vel.device, dtype=torch.float32)
                                       for k in (n[2], n[1], n[0])], indexing="ij")
            blob = torch.exp(-((x - n[0] / 3) ** 2 + (y - n[1] / 2) ** 2 + (z - n[2] / 2) ** 2) / 50.0)
            vel = vel / torch.sqrt(1.0 + (scale - 1.0) * blob)      # m = 1/v^2 times (1 + a blob)
        rec = np.array([(2, j, k) for j in range(2, n[1] - 2, 4) for k in range(2, n[2] - 2, 4)])
        shots.append(Shot(n=n, dx=DX, vel=vel, src=(3, n[1] // 2, n[2] // 2), rec=rec, amp=2.0,
                          sponge=6, dobs=None if dobs is None else dobs[i]))
    return shots


def dt_of():
    from hpcscan_b200.modeling import stable_dt
    return stable_dt(ORDER, DX, 2700.0)


def oracle_inputs(batch, i):
    """FP64 copies of exactly what shot i of the batch computes with."""
    st = batch.states[i]
    lay = st.lay
    C = st.coef.double().cpu().numpy()
    g = [t.cpu().numpy() for t in st.sponge]
    G = (g[0][None, None, :] * g[1][None, :, None]) * g[2][:, None, None]     # FP32, (g1 g2) g3
    G = G.reshape(-1).astype(np.float64)
    inv2 = tuple(float(np.float32(1.0 / DX) * np.float32(1.0 / DX)) for _ in range(3))
    return lay, C, G, st.src_flat, st.rec.cpu().numpy(), inv2, st.wavelet.double().cpu().numpy()


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def test_forward_traces_match_fp64_oracle(gpu):
    from hpcscan_b200.modeling import Batch
    from oracle import oracle
    b = Batch(make_shots(gpu), ORDER, dt_of(), NT, F0)
    b.forward()
    gpu.cuda.synchronize()
    for i in range(2):
        lay, C, G, src, rec, inv2, wav = oracle_inputs(b, i)
        want = oracle.model_forward(lay, C, G, src, 2.0, wav, rec, inv2)
        got = b.traces(i).double().cpu().numpy()
        assert np.abs(want).max() > 0
        assert rel(got, want) < 2e-5, rel(got, want)
    b.close()


def observed(gpu, sizes=((36, 30, 40), (28, 36, 24))):
    from hpcscan_b200.modeling import Batch
    b = Batch(make_shots(gpu, sizes, scale=1.25), ORDER, dt_of(), NT, F0)
    b.forward()
    gpu.cuda.synchronize()
    d = [b.traces(i).clone() for i in range(len(sizes))]
    b.close()
    return d


def test_gradient_matches_fp64_oracle_and_is_checkpoint_invariant(gpu):
    from hpcscan_b200.modeling import Batch
    from oracle import oracle
    dobs = observed(gpu)
    grads = {}
    for k in (7, NT):
        b = Batch(make_shots(gpu, dobs=dobs), ORDER, dt_of(), NT, F0, gradient=True, checkpoint=k)
        b.forward()
        b.backward()
        gpu.cuda.synchronize()
        grads[k] = [b.states[i].grad.clone() for i in range(2)]
        if k == 7:
            for i in range(2):
                lay, C, G, src, rec, inv2, wav = oracle_inputs(b, i)
                J, g = oracle.model_gradient(lay, C, G, src, 2.0, wav, rec, inv2,
                                             dobs[i].double().cpu().numpy(), b.dt)
                got = b.states[i].grad.double().cpu().numpy()
                assert np.abs(g).max() > 0
                assert rel(got, g) < 1e-3, rel(got, g)
                assert b.misfit(i) == pytest.approx(J, rel=1e-4)
        b.close()
    for i in range(2):
        assert gpu.equal(grads[7][i], grads[NT][i])


def test_batch_equals_single_shots_and_graph_equals_eager(gpu):
    from hpcscan_b200.modeling import Batch, run_graph
    dobs = observed(gpu)
    b = Batch(make_shots(gpu, dobs=dobs), ORDER, dt_of(), NT, F0, gradient=True, checkpoint=11)
    b.forward()
    b.backward()
    gpu.cuda.synchronize()
    both = [(b.traces(i).clone(), b.states[i].grad.clone()) for i in range(2)]
    # the same schedule captured in one CUDA graph and replayed
    g = run_graph(lambda s: (b.forward(s), b.backward(s)))
    for st in b.states:
        st.grad.zero_()
        st.traces.zero_()
    g.replay()
    gpu.cuda.synchronize()
    for i in range(2):
        assert gpu.equal(b.traces(i), both[i][0]) and gpu.equal(b.states[i].grad, both[i][1])
    del g
    b.close()
    for i, n in enumerate(((36, 30, 40), (28, 36, 24))):
        one = Batch(make_shots(gpu, (n,), seed=i, dobs=[dobs[i]]), ORDER, dt_of(), NT, F0,
                    gradient=True, checkpoint=11)
        one.forward()
        one.backward()
        gpu.cuda.synchronize()
        assert gpu.equal(one.traces(0), both[i][0])
        assert gpu.equal(one.states[0].grad, both[i][1])
        one.close()


def test_survey_gradient_is_the_sum_of_the_shards(gpu):
    """The shot-parallel split: shots 0 and 2 on one 'rank', shot 1 on another, each its own
    batch; the survey gradient (hpcscan_b200.shots) of the shards, summed, equals the per-shot
    gradients of one batch of all three shots, summed in the same order (bit for bit: shots are
    independent in a batch, and the sums are the same FP32 additions)."""
    from hpcscan_b200.modeling import Batch
    from hpcscan_b200.shots import my_shots, sum_gradients, survey_gradient
    n = (30, 28, 26)
    sizes = (n, n, n)
    ref = Batch(make_shots(gpu, sizes, seed=3), ORDER, dt_of(), NT, F0)
    ref.forward()
    gpu.cuda.synchronize()
    dobs = [ref.traces(i).clone() * 1.01 for i in range(3)]
    ref.close()
    full = Batch(make_shots(gpu, sizes, seed=3, dobs=dobs), ORDER, dt_of(), NT, F0, gradient=True,
                 checkpoint=11)
    full.forward()
    full.backward()
    gpu.cuda.synchronize()
    per_shot = [full.gradient_of(i).clone() for i in range(3)]
    assert gpu.equal(survey_gradient(full), (per_shot[0] + per_shot[1]) + per_shot[2])
    full.close()
    parts = [my_shots([1.0] * 3, r, 2) for r in range(2)]
    assert parts == [[0, 2], [1]]
    shots = make_shots(gpu, sizes, seed=3, dobs=dobs)
    shard_sums = []
    for part in parts:
        b = Batch([shots[i] for i in part], ORDER, dt_of(), NT, F0, gradient=True, checkpoint=11)
        b.forward()
        b.backward()
        gpu.cuda.synchronize()
        for j, i in enumerate(part):
            assert gpu.equal(b.gradient_of(j), per_shot[i])
        shard_sums.append(survey_gradient(b))
        b.close()
    # the all-reduce of two ranks adds the two shard sums
    assert gpu.equal(sum_gradients(shard_sums), (per_shot[0] + per_shot[2]) + per_shot[1])


def test_gpu_gradient_matches_central_differences(gpu):
    """The GPU adjoint gradient against central differences of the GPU misfit (FP32 forward
    runs): J(m +- delta) along delta = 1e-3 max|m| g / max|g| per shot (m = 1/v^2 on the inner
    points), (J+ - J-) / 2 against sum(g delta). Along the gradient the change of J stands well
    above the FP32 rounding of the traces; agreement within 2 %."""
    torch = gpu
    from hpcscan_b200.modeling import Batch
    dobs = observed(gpu)
    shots = make_shots(gpu, dobs=dobs)
    b = Batch(shots, ORDER, dt_of(), NT, F0, gradient=True, checkpoint=11)
    b.forward()
    b.backward()
    torch.cuda.synchronize()
    grads = [b.gradient_of(i).double() for i in range(2)]
    b.close()
    deltas, an = [], 0.0
    for sh, g in zip(shots, grads):
        m0 = 1.0 / sh.vel.double() ** 2
        d = 1e-3 * float(m0.abs().max()) * g / float(g.abs().max())
        deltas.append(d)
        an += float((g * d).sum())

    def misfit(sign):
        import dataclasses
        pert = [dataclasses.replace(sh, vel=(1.0 / torch.sqrt(1.0 / sh.vel.double() ** 2 + sign * d))
                                    .float().contiguous())
                for sh, d in zip(shots, deltas)]
        f = Batch(pert, ORDER, dt_of(), NT, F0)
        f.forward()
        torch.cuda.synchronize()
        J = sum(0.5 * float(((f.traces(i).double() - sh.dobs.double()) ** 2).sum())
                for i, sh in enumerate(shots))
        f.close()
        return J

    fd = (misfit(+1.0) - misfit(-1.0)) / 2.0
    assert an > 0.0
    assert fd == pytest.approx(an, rel=2e-2), (fd, an)


def test_dot_product_of_the_gpu_forward_adjoint_pair(gpu):
    """The GPU forward and adjoint kernels are each other's transpose: with d = F(amp s) the
    traces of the forward pass and r a random residual injected by the adjoint pass,
    <d, r> = <amp s, w_src> / C(src), w_src[n] = w[n+1](src) read after each adjoint step.
    FP32 kernels, FP64 sums; two shots of different sizes in one batch."""
    import ctypes

    from hpcscan_b200 import _lib
    from hpcscan_b200.modeling import Batch
    b = Batch(make_shots(gpu), ORDER, dt_of(), NT, F0)
    b.forward()
    gpu.cuda.synchronize()
    d = [b.traces(i).clone() for i in range(2)]
    b.close()
    rng = np.random.default_rng(11)
    r = [torch_randn(gpu, x.shape, rng) for x in d]
    # the adjoint pass alone, driven by the residual r: traces = r, dobs = 0
    a = Batch(make_shots(gpu, dobs=[gpu.zeros_like(x) for x in d]), ORDER, dt_of(), NT, F0,
              gradient=True, checkpoint=NT)
    for i, st in enumerate(a.states):
        st.traces.copy_(r[i])                                   # residual row k-1 = traces - dobs
        a._zero(st.adj, None)
    wsrc = [gpu.zeros(NT, dtype=gpu.float32, device="cuda:0") for _ in range(2)]
    idx = [gpu.tensor([st.src_flat], dtype=gpu.int64, device="cuda:0") for st in a.states]
    s = ctypes.c_void_p(gpu.cuda.current_stream().cuda_stream)
    for k in range(NT, 0, -1):
        scur = (NT - k) % 2
        _lib.call("b200_batch_adjoint_step", a.handle, k, scur, s)
        for i, st in enumerate(a.states):                       # w[k](src) -> w_src[k - 1]
            f = _lib.Field(ctypes.c_void_p(st.adj[1 - scur].data_ptr()), _lib.B200_F32, 1.0)
            _lib.call("b200_gather_points", f, ctypes.c_void_p(idx[i].data_ptr()), 1,
                      ctypes.c_void_p(wsrc[i][k - 1:].data_ptr()), 1, s)
    gpu.cuda.synchronize()
    for i, st in enumerate(a.states):
        lhs = float((d[i].double() * r[i].double()).sum())
        csrc = float(st.coef[st.src_flat])
        rhs = float((2.0 * st.wavelet.double() * wsrc[i].double()).sum()) / csrc
        assert abs(lhs) > 0
        assert rhs == pytest.approx(lhs, rel=1e-4), (i, lhs, rhs)
    a.close()


def torch_randn(torch, shape, rng):
    return torch.from_numpy(rng.standard_normal(tuple(shape)).astype(np.float32)).to("cuda:0")


def test_survey_gradient_equals_sum_of_shot_gradients(gpu):
    """Shots on one grid (survey=True): the survey gradient accumulated in one stencil-free pass
    per step (C Lap p[n] from p[n+1], p[n], p[n-1] by the forward recursion) equals the sum of
    the per-shot gradients (stencil pass per shot) to FP32 rounding, matches the FP64 oracle's
    summed gradients, and is bit-identical across checkpoint intervals."""
    from hpcscan_b200.modeling import Batch
    from hpcscan_b200.shots import survey_gradient
    from oracle import oracle
    sizes = ((36, 30, 40), (36, 30, 40), (36, 30, 40))
    dobs = observed(gpu, sizes)
    shots = lambda: make_shots(gpu, sizes, dobs=dobs)                              # noqa: E731
    ref = Batch(shots(), ORDER, dt_of(), NT, F0, gradient=True, checkpoint=7)
    ref.forward()
    ref.backward()
    want = survey_gradient(ref).double()
    oracle_sum = None
    for i in range(len(sizes)):
        lay, C, G, src, rec, inv2, wav = oracle_inputs(ref, i)
        _, g = oracle.model_gradient(lay, C, G, src, 2.0, wav, rec, inv2,
                                     dobs[i].double().cpu().numpy(), ref.dt)
        g = np.asarray(g).reshape(lay.n3, lay.n2, lay.n1)[
            lay.a3.inner_start:lay.a3.inner_end + 1, lay.a2.inner_start:lay.a2.inner_end + 1,
            lay.a1.inner_start:lay.a1.inner_end + 1]
        oracle_sum = g if oracle_sum is None else oracle_sum + g
    ref.close()
    got = {}
    for k in (7, 50):
        b = Batch(shots(), ORDER, dt_of(), NT, F0, gradient=True, checkpoint=k, survey=True)
        b.forward()
        b.backward()
        got[k] = survey_gradient(b).clone()
        b.close()
    assert gpu.equal(got[7], got[50])
    g = got[7].double()
    assert rel(g.cpu().numpy(), want.cpu().numpy()) < 1e-4, rel(g.cpu().numpy(), want.cpu().numpy())
    assert rel(g.cpu().numpy(), oracle_sum) < 1e-3, rel(g.cpu().numpy(), oracle_sum)
