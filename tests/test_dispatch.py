"""The dispatcher and cost model (crates/spatial-query/src/dispatch.rs) with
this library as the Gpu backend.

With the crate's own GPU constants the restated model makes the crate's
decisions (the selection matrix of tests/dispatch.rs:160-276, stub backends
as there); with the B200 constants measured for this library the CPU/GPU
crossover moves from the crate's measured 256..2048-ray band at 100,000
leaves down to a few dozen rays; and the CUDA backend, chosen by the
dispatcher, returns the oracle's hits (tests/dispatch.rs:278-298).
"""
import numpy as np
import pytest

import oracle as O
import spatial_query_b200 as sq
from gpu_util import assert_same_nearest
from spatial_query_b200 import dispatch as D
from spatial_query_b200 import scenes

K = D.BackendKind


class Stub:
    def __init__(self, kind, cost, needs_device):
        self._kind, self._cost, self._dev = kind, cost, needs_device

    def kind(self):
        return self._kind

    def can_serve(self, ctx):
        return ctx.device_available or not self._dev

    def estimate_cost(self, ctx):
        return self._cost(ctx)

    def raycast_nearest_batch(self, rays, max_toi, **kw):
        return self._kind


def full(gpu=D.REFERENCE_GPU):
    d = D.Dispatcher(Stub(K.CPU, D.cpu_batch_us, False))
    d.register(Stub(K.DRAW_PASS, D.draw_pass_batch_us, True))
    d.register(Stub(K.GPU, lambda c: D.gpu_batch_us(c, gpu), True))
    return d


def test_deterministic_request_pins_cpu():
    ctx = D.QueryContext(100_000, 100_000, 100_000).with_device(True).deterministic(True)
    assert full().select(ctx) == K.CPU
    assert full(D.B200).select(ctx) == K.CPU


def test_no_device_falls_back_to_cpu():
    assert full().select(D.QueryContext(1, 1, 100_000).with_device(False)) == K.CPU


@pytest.mark.parametrize("gpu", [D.REFERENCE_GPU, D.B200])
def test_single_view_large_scene_picks_draw_pass(gpu):
    d = full(gpu)
    assert d.select(D.QueryContext(1, 1, 100_000).with_device(True)) == K.DRAW_PASS
    assert d.select(D.QueryContext(5_000, 1, 100_000).with_device(True)) == K.DRAW_PASS


@pytest.mark.parametrize("gpu", [D.REFERENCE_GPU, D.B200])
def test_scattered_large_batch_picks_gpu(gpu):
    assert full(gpu).select(D.QueryContext(100_000, 100_000, 100_000).with_device(True)) == K.GPU


def test_cpu_only_dispatcher_selects_cpu():
    d = D.Dispatcher(Stub(K.CPU, D.cpu_batch_us, False))
    assert d.select(D.QueryContext(1, 1, 100_000).with_device(True)) == K.CPU


def test_force_override_wins_over_everything():
    d = full()
    d.force(K.GPU)
    ctx = D.QueryContext(1, 1, 10).deterministic(True)
    assert d.select(ctx) == K.GPU
    d.force(None)
    assert d.select(ctx) == K.CPU


def test_crate_constants_cross_over_in_the_measured_band():
    d = full()
    scattered = lambda b, n: D.QueryContext(b, b, n).with_device(True)
    assert d.select(scattered(64, 100_000)) == K.CPU
    assert d.select(scattered(8_000, 100_000)) == K.GPU
    assert 256 <= D.crossover_batch(100_000, D.REFERENCE_GPU) <= 2048


def test_b200_constants_move_the_crossover_down():
    ref = D.crossover_batch(100_000, D.REFERENCE_GPU)
    b200 = D.crossover_batch(100_000, D.B200)
    assert b200 <= ref // 8
    # a 256-ray batch of cheap leaves now amortises the GPU's fixed cost
    assert full(D.B200).select(D.QueryContext(256, 256, 100_000).with_device(True)) == K.GPU
    assert full(D.REFERENCE_GPU).select(D.QueryContext(256, 256, 100_000).with_device(True)) == K.CPU


@pytest.mark.parametrize("gpu", [D.REFERENCE_GPU, D.B200])
def test_expensive_field_leaves_route_to_gpu_sooner(gpu):
    for leaves in (1_000, 100_000):
        cheap = D.crossover_batch(leaves, gpu, hint=1.0)
        field = D.crossover_batch(leaves, gpu, hint=30.0)
        assert field < cheap or field == 2


def test_reference_field_case():
    cheap = D.QueryContext(256, 256, 100_000).with_device(True)
    assert full().select(cheap) == K.CPU
    assert full().select(cheap.with_narrow_cost(30.0)) == K.GPU


@pytest.mark.gpu
def test_cuda_backend_agrees_with_oracle():
    ctx = sq.Context(0)
    rng = scenes.Rng(0xD15_0A7C)
    n = 2000
    balls = np.ascontiguousarray(np.concatenate([rng.range(-40.0, 40.0, (n, 3)), np.ones((n, 1))], axis=1),
                                 dtype=np.float32)
    geom = sq.Geometry("balls", 3, balls)
    scene = sq.DeviceBvh(ctx, sq.HostBvh.build(geom), geom)
    o = rng.range(-50.0, 50.0, (500, 3)).astype(np.float32)
    rays = np.ascontiguousarray(np.concatenate([o, scenes.normalize_rows(-o)], axis=1), dtype=np.float32)
    oracle_scene = O.Scene("balls", 3, balls)

    class OracleCpu:
        def kind(self):
            return K.CPU

        def can_serve(self, c):
            return True

        def estimate_cost(self, c):
            return D.cpu_batch_us(c)

        def raycast_nearest_batch(self, r, max_toi, **kw):
            return oracle_scene.nearest(r, max_toi)

    d = D.Dispatcher(OracleCpu())
    d.register(D.CudaBackend(scene))
    kind, hits = d.raycast_nearest_batch(rays, 500.0, D.QueryContext(0, len(rays), n).with_device(True))
    assert kind == K.GPU
    assert_same_nearest(oracle_scene.nearest(rays, 500.0), hits, label="dispatched GPU backend")
    scene.close()
    ctx.close()
