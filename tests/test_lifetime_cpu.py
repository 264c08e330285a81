"""Handle lifetimes of the Python facade, on a recording fake of the C library (no GPU):
a context closed while TransportMaps built on it are alive frees their device maps first
(otm_destroy requires every otm_map of the context destroyed before it), and a map
released that way is not freed again when it is collected."""

import gc

import numpy as np


class FakeLib:
    def __init__(self):
        self.calls = []
        self.next = 100

    def otm_create(self, device, h):
        h._obj.value = 1
        self.calls.append(("create",))
        return 0

    def otm_destroy(self, h):
        self.calls.append(("destroy", h.value))
        return 0

    def otm_map_create(self, ctx, n, fwd, dens, h):
        self.next += 1
        h._obj.value = self.next
        self.calls.append(("map_create", self.next))
        return 0

    def otm_map_destroy(self, m):
        self.calls.append(("map_destroy", m.value))
        return 0

    def otm_map_init_inverse(self, m):
        return 0


def test_close_releases_maps_first(monkeypatch):
    from otmap_b200 import native as N
    from otmap_b200 import otmap as ot

    fake = FakeLib()
    monkeypatch.setattr(N, "lib", lambda: fake)
    ctx = N.Context(0)
    n = 4
    maps = [ot.TransportMap(n, ot.grid_vertices(n), np.ones(n * n), context=ctx) for _ in range(2)]
    for m in maps:
        m.init_inverse()
    unused = ot.TransportMap(n, ot.grid_vertices(n), np.ones(n * n), context=ctx)  # no device map
    ctx.close()
    names = [c[0] for c in fake.calls]
    assert names == ["create", "map_create", "map_create", "map_destroy", "map_destroy", "destroy"]
    del maps, unused
    gc.collect()
    assert [c[0] for c in fake.calls].count("map_destroy") == 2
    ctx.close()  # idempotent
    assert [c[0] for c in fake.calls].count("destroy") == 1


def test_collected_map_destroyed_once(monkeypatch):
    from otmap_b200 import native as N
    from otmap_b200 import otmap as ot

    fake = FakeLib()
    monkeypatch.setattr(N, "lib", lambda: fake)
    ctx = N.Context(0)
    m = ot.TransportMap(2, ot.grid_vertices(2), np.ones(4), context=ctx)
    m.init_inverse()
    del m
    gc.collect()
    ctx.close()
    assert [c[0] for c in fake.calls] == ["create", "map_create", "map_destroy", "destroy"]
