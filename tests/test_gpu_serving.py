"""GPU tests of the serving path: re-meshing a live context, CUDA-graph replay
of the solver's inner operators, and the serving loop (a request gives the
same result alone and in a mix of concurrent requests)."""
import numpy as np
import pytest

from baemm_b200 import APPLY_FP32, APPLY_TC, Helmholtz_CUDA, WaveType, meshes
from baemm_b200.serving import SolveRequest, SolveServer, make_stream, summarize
from tests.helpers import crandn, relerr

pytestmark = pytest.mark.gpu


def _apply(H, B, kap, coeff, wc, wcs):
    C = np.zeros_like(B)
    H.ApplyBoundaryOperators_PL(1.0, B, 0.0, C, kap, coeff, wc, wcs)
    return C


def test_set_mesh_matches_a_fresh_context():
    """A context re-meshed (to a larger, then a smaller mesh) computes exactly
    what a context created on that mesh computes."""
    meas = meshes.fibonacci_sphere(16)
    small = meshes.sh_perturbed_sphere(2, 4, 0.1, seed=1)
    large = meshes.sh_perturbed_sphere(3, 4, 0.1, seed=2)
    kap = [3.0]
    coeff = np.array([[0.5, -3j, 1.0, 0.25]])
    with Helmholtz_CUDA(*small, meas) as H:
        for coords, tris in (large, small):
            H.SetMesh(coords, tris)
            B = crandn(np.random.default_rng(coords.shape[0]), coords.shape[0], 16)
            with Helmholtz_CUDA(coords, tris, meas) as F:
                ref = _apply(F, B, kap, coeff, 16, 16)
                assert np.array_equal(F.Areas(), H.Areas())
            assert H.VertexCount() == coords.shape[0]
            assert np.array_equal(_apply(H, B, kap, coeff, 16, 16), ref)


@pytest.mark.parametrize("mode", [APPLY_FP32, APPLY_TC])
def test_graphs_give_the_same_solve(mode):
    """FarField with the GMRES apply and the CG mass inverse replayed as CUDA
    graphs equals the solve without graphs (same kernels, same order)."""
    coords, tris = meshes.icosphere(3)
    meas = meshes.fibonacci_sphere(32)
    inc = meshes.fibonacci_sphere(16)
    kap = np.array([4.0])
    with Helmholtz_CUDA(coords, tris, meas) as H:
        H.SetApplyMode(mode)
        F0 = np.zeros((32, 16), complex)
        H.FarField(kap, inc, F0, WaveType.Plane, 1e-8, 1e-8)
        H.SetGraphs(True)
        for _ in range(2):
            F1 = np.zeros((32, 16), complex)
            H.FarField(kap, inc, F1, WaveType.Plane, 1e-8, 1e-8)
            assert relerr(F1, F0) < 1e-12
        captures, replays = H.GraphStats()
        assert captures > 0 and replays > captures


def _requests(n, seed):
    reqs = make_stream(n, rate=0.0, levels=(2, 3), kappa_range=(1.0, 6.0), rhs_range=(1, 40), degree=4,
                       seed=seed)
    for r in reqs:
        r.gmres_tol = 1e-8
    return reqs


def test_result_is_the_same_alone_and_in_the_mix():
    """Each request's far field served concurrently with others equals the
    same request served alone (tolerance 1e-10: the kernels are deterministic;
    only the interleaving of other requests' work differs)."""
    meas = meshes.fibonacci_sphere(24)
    reqs = _requests(10, seed=7)
    with SolveServer(meas, slots=4, graphs=True) as srv:
        mix = srv.run(reqs, realtime=False)
        assert srv.scheduler.peak_running > 1
    for r in reqs[:4]:
        with SolveServer(meas, slots=1, graphs=False) as alone:
            one = alone.run([SolveRequest(r.rid, r.coords, r.triangles, r.kappa, r.directions,
                                          gmres_tol=r.gmres_tol)], realtime=False)
        assert one[r.rid].converged and mix[r.rid].converged
        assert relerr(mix[r.rid].far_field, one[r.rid].far_field) < 1e-10
    s = summarize(mix)
    assert s["requests"] == 10 and s["converged"] == 10


def test_served_tensor_core_matches_plain():
    """Served tensor-core solves agree with plain FP32 solves at the solve
    tolerance (the accuracy the serving comparison is stated at)."""
    meas = meshes.fibonacci_sphere(24)
    reqs = _requests(4, seed=11)
    with SolveServer(meas, slots=2, apply_mode=APPLY_TC) as a, SolveServer(meas, slots=1, apply_mode=APPLY_FP32,
                                                                          graphs=False) as b:
        ra = a.run(reqs, realtime=False)
        rb = b.run(reqs, realtime=False)
    for r in reqs:
        assert relerr(ra[r.rid].far_field, rb[r.rid].far_field) < 1e-5


def test_packed_solves_are_the_same_alone_and_packed():
    """Two contexts on one packer (two meshes), each solving a BoundaryPotential
    in its own thread: the GMRES applies of the two solves share launches, and
    each solution equals the same solve run alone on the packer bit for bit
    (whole target blocks, the same sums); the packed apply meets the bar of the
    FP64 oracle."""
    import threading

    from baemm_b200 import APPLY_TC, Packer
    from oracle import oracle as O

    meshes_ = [meshes.icosphere(2), meshes.icosphere(3)]
    kap = np.array([3.0])
    rng = np.random.default_rng(3)
    waves = [crandn(rng, c.shape[0], 16) for c, _ in meshes_]
    with Packer(0, max_wait_us=100000) as P:
        Hs = [Helmholtz_CUDA(c, t, np.eye(3)) for c, t in meshes_]
        try:
            for H in Hs:
                H.SetApplyMode(APPLY_TC)
                H.SetPacker(P)

            def solve(q):
                phi = np.zeros_like(waves[q])
                Hs[q].BoundaryPotential(kap, np.zeros((1, 4), complex), waves[q], phi, 16, 1e-10, 1e-10)
                return phi

            alone = [solve(0), solve(1)]        # one at a time: every launch carries one problem
            before = P.stats()
            assert before["problems"] == before["launches"]
            outs = [None, None]
            barrier = threading.Barrier(2)

            def run(q):
                barrier.wait()
                outs[q] = solve(q)

            th = [threading.Thread(target=run, args=(q,)) for q in range(2)]
            for t in th:
                t.start()
            for t in th:
                t.join()
            after = P.stats()
            for q in range(2):
                assert np.array_equal(outs[q], alone[q])
            assert after["problems"] - before["problems"] > after["launches"] - before["launches"]
            # one packed apply against the FP64 oracle
            coeff = np.array([[0.5, -3j, 1.0, 0.0]])
            c, t = meshes_[1]
            B = crandn(rng, c.shape[0], 16)
            Cg, Co = np.zeros_like(B), np.zeros_like(B)
            Hs[1].ApplyBoundaryOperators_PL(1.0, B, 0.0, Cg, kap, coeff, 16, 16)
            O.Oracle(c, t, np.eye(3), precision=64).ApplyBoundaryOperators_PL(1.0, B, 0.0, Co, kap, coeff, 16, 16)
            assert relerr(Cg, Co) < 1e-5
        finally:
            for H in Hs:
                H.SetPacker(None)
                H.close()


def test_packed_problems_with_different_wave_shapes():
    """Two solves of one packing class whose chunk groups per unit come from
    different settings (64 columns tuned to 2 chunks per unit, 32 columns with
    the automatic choice, also 2) share packed launches in either order, and
    each solution equals the same solve run alone bit for bit."""
    import threading

    from baemm_b200 import APPLY_TC, Packer, _capi

    meshes_ = [meshes.icosphere(2), meshes.icosphere(3)]
    kaps = [np.array([2.0, 3.0, 4.0, 5.0]), np.array([3.0, 6.0])]
    rng = np.random.default_rng(11)
    waves = [crandn(rng, c.shape[0], 16 * len(ka)) for (c, _), ka in zip(meshes_, kaps)]
    with Packer(0, max_wait_us=100000) as P:
        Hs = [Helmholtz_CUDA(c, t, np.eye(3)) for c, t in meshes_]
        try:
            Hs[0].SetTuning(_capi.TUNE_TC_CHUNKS, 2)
            for H in Hs:
                H.SetApplyMode(APPLY_TC)
                H.SetPacker(P)

            def solve(q):
                phi = np.zeros_like(waves[q])
                Hs[q].BoundaryPotential(kaps[q], np.zeros((len(kaps[q]), 4), complex), waves[q], phi, 16,
                                        1e-10, 1e-10)
                return phi

            alone = [solve(0), solve(1)]
            before = P.stats()
            outs = [[], []]
            barrier = threading.Barrier(2)
            errors = []

            def run(q):
                try:
                    for _ in range(2):
                        barrier.wait()
                        outs[q].append(solve(q))
                except Exception as e:   # surfaced below
                    errors.append(e)
                    barrier.abort()

            th = [threading.Thread(target=run, args=(q,)) for q in range(2)]
            for t in th:
                t.start()
            for t in th:
                t.join()
            assert not errors, errors
            after = P.stats()
            for q in range(2):
                for phi in outs[q]:
                    assert np.array_equal(phi, alone[q])
            assert after["problems"] - before["problems"] > after["launches"] - before["launches"]
        finally:
            for H in Hs:
                H.SetPacker(None)
                H.close()


def test_packed_server_same_alone_and_in_the_mix():
    """The packing server: each request's far field alone equals the same
    request in a concurrent mix (1e-10), and the mix's applies shared launches."""
    meas = meshes.fibonacci_sphere(24)
    reqs = _requests(8, seed=5)
    with SolveServer(meas, slots=4, graphs=True, pack=True, pack_wait_us=5000) as srv:
        mix = srv.run(reqs, realtime=False)
        st = srv.pack_stats()
        assert srv.scheduler.peak_running > 1
    assert st["launches"] > 0 and st["problems"] > st["launches"]   # some launches carried several problems
    for r in reqs[:3]:
        with SolveServer(meas, slots=1, graphs=True, pack=True) as alone:
            one = alone.run([SolveRequest(r.rid, r.coords, r.triangles, r.kappa, r.directions,
                                          gmres_tol=r.gmres_tol)], realtime=False)
        assert one[r.rid].converged and mix[r.rid].converged
        assert relerr(mix[r.rid].far_field, one[r.rid].far_field) < 1e-10
