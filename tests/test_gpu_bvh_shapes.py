"""Primary hits on scenes whose BVH takes unusual shapes, CUDA against the
oracle bit for bit (triangle ids and distances): triangle counts around the
8-wide node's and the three-triangle leaf's capacities, where the SAH-optimal
collapse decides between leaves and internal children; many identical
triangles (equal boxes, ties resolved by the smaller primitive index); a
dense cluster of tiny triangles beside large ones; and long thin slivers."""
import numpy as np
import pytest

from hdcodex_b200 import Material, Mesh, PathTracer, Scene, workloads

pytestmark = pytest.mark.gpu

W = H = 64


def scene_of(triangles):
    t = np.asarray(triangles, np.float32).reshape(-1, 3, 3)
    s = Scene(revision=1)
    s.meshes.append(Mesh(id="/tris", positions=t.ravel().tolist(), indices=list(range(3 * len(t))),
                         material_id="/m"))
    s.materials.append(Material(id="/m", base_color=[0.7, 0.7, 0.7]))
    return s


def random_triangles(n, seed, size=0.3):
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-1.0, 1.0, (n, 1, 3))
    return centres + rng.uniform(-size, size, (n, 3, 3))


def shapes():
    out = {f"random{n}": random_triangles(n, n) for n in (1, 2, 3, 4, 7, 8, 9, 24, 25, 26, 200)}
    one = random_triangles(1, 99)[0]
    out["identical64"] = np.repeat(one[None], 64, axis=0)
    rng = np.random.default_rng(5)
    tiny = rng.uniform(-1e-4, 1e-4, (300, 3, 3)) + np.array([0.2, 0.1, 0.0])
    out["cluster"] = np.concatenate([tiny, random_triangles(20, 6, size=0.8)])
    x = np.linspace(-1.0, 1.0, 101)
    slivers = [[[x[i], -1.0, 0.3 * np.sin(3 * x[i])], [x[i + 1], -1.0, 0.3 * np.sin(3 * x[i + 1])],
                [x[i], 1.0, 0.3 * np.sin(3 * x[i])]] for i in range(100)]
    out["slivers"] = np.asarray(slivers)
    return out


SHAPES = shapes()


@pytest.mark.parametrize("name", sorted(SHAPES))
def test_primary_hits_match_oracle(oracle_lib, name):
    scene = scene_of(SHAPES[name])
    cam = workloads.look_at_camera((0.3, 0.4, 3.5), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 45.0, 1.0)
    o = oracle_lib.OracleTracer()
    o.set_scene(scene)
    with PathTracer(0) as t:
        t.set_scene(scene)
        for sample in (0, 5):
            ref_p, ref_t = o.trace_primary(cam, W, H, sample)
            got_p, got_t = t.trace_primary(cam, W, H, sample)
            assert (ref_p != 0xFFFFFFFF).any()
            assert np.array_equal(got_p, ref_p)
            assert np.array_equal(got_t.view(np.uint32), ref_t.view(np.uint32))
