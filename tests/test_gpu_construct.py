"""Solver construction: the split node orders found on the device, and the device memory a construction reuses.

A node's update reads the same 27 values in the same order whatever the internal numbering, so the fields of any
node order, mapped back to the lattice's order, are bit-identical to those of the lattice's own order.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from cerebrosim_b200 import cases, lbm, workloads  # noqa: E402

NU = (0.55 - 0.5) / 3.0


@pytest.fixture(scope="module")
def pipe():
    c = cases.case("open_pipe_R24_L192")
    return cases.plug_inlet(lbm.build_lattice(**cases.lattice_args(c)))


def solver(lat, **kw):
    s = lbm.Solver(lat, NU, model="regularised", **kw)
    s.set_drive([0.02, 0.0, 0.01], period=4000)
    s.set_outlet_pressure([0.0])
    return s


@pytest.mark.parametrize("order", ["split", "boundary-first"])
@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_split_orders_on_the_device(pipe, order, storage):
    """The C-based split orders (nodes with a boundary link last, or first) are computed on the device from the
    uploaded table; each is the host's node_order, and 300 steps on it give the C order's fields bit for bit."""
    a = solver(pipe, storage=storage)
    b = solver(pipe, storage=storage, order=order)
    assert np.array_equal(b.perm.cpu().numpy(), lbm.node_order(pipe, order))
    n = pipe["nbr"].shape[1]
    n_bnd = int((np.asarray(pipe["nbr"]) < 0).any(0).sum())
    plain = slice(0, n - n_bnd) if order == "split" else slice(n_bnd, n)
    assert int((b.inl[plain] != 0).sum()) == 0          # the inlet cells are among the boundary nodes
    for s in (a, b):
        s.run(300, chunk=100)
    pa, ua = a.fields()
    pb, ub = b.fields()
    assert a.ok() and b.ok()
    assert np.array_equal(pa, pb) and np.array_equal(ua, ub)


@pytest.mark.parametrize("order", ["split", "boundary-first"])
def test_split_orders_from_host_tables(pipe, order):
    """From NumPy tables (no device copy in the lattice) the device-computed order is the same."""
    host = {k: v for k, v in pipe.items() if k != "_dev"}
    s = solver(host, order=order)
    assert np.array_equal(s.perm.cpu().numpy(), lbm.node_order(pipe, order))


@pytest.mark.parametrize("order", ["axis", "split", "axis-split", "boundary-first", "axis-boundary-first"])
def test_device_orders_equal_host_orders(order):
    """Every order the solver computes on the device is the host's node_order, on a generated artery (whose axis
    order differs from its C order), from device tables and from host tables (coordinates uploaded)."""
    lat = workloads.lattice(workloads.stenosed_vessel(3), 0.1)
    host_perm = lbm.node_order(lat, order)
    assert host_perm is not None
    host = {k: lat[k] for k in list(lat) + ["nbr", "q", "uin", "coords"] if k != "_dev"}   # host copies read
    for tables in (lat, host):
        s = lbm.Solver(tables, NU, model="regularised", order=order)
        assert s.perm is not None and np.array_equal(s.perm.cpu().numpy(), host_perm)


def test_constructions_reuse_device_memory(pipe):
    """A Solver allocates its tables and populations on the caller's stream, so the next Solver built after it is
    freed takes the same cached blocks: the allocator's reserve does not grow by a lattice's footprint."""
    torch.cuda.synchronize()
    s = solver(pipe)
    s.run(10)
    footprint = sum(t.numel() * t.element_size() for t in (*s.f, *s.vel, s.rho, s.om, s.lcode))
    del s
    torch.cuda.synchronize()
    r0 = torch.cuda.memory_reserved()
    for _ in range(3):
        s = solver(pipe)
        s.run(10)
        assert s.ok()
        del s
        torch.cuda.synchronize()
    grown = torch.cuda.memory_reserved() - r0
    assert footprint > 64 << 20
    assert grown < footprint // 4, f"reserve grew by {grown >> 20} MiB over three constructions"


@pytest.mark.parametrize("order", ["c", "boundary-first"])
def test_pinned_host_tables(pipe, order):
    """From pinned host tensors (the end-to-end path: two of the three tables are copied on a side stream while the
    set-up works on the first) the solver's tables and fields are those built from the device tables."""
    host = {k: v for k, v in pipe.items() if k != "_dev"}
    for k in ("nbr", "q", "uin"):
        host[k] = torch.from_numpy(np.ascontiguousarray(pipe[k])).pin_memory()
    a = solver(pipe, order=order)
    b = solver(host, order=order)
    for name in ("lcode", "segdelta", "irr", "gnode", "ginfo", "gq", "uin", "om"):
        assert torch.equal(getattr(a, name), getattr(b, name)), name
    for s in (a, b):
        s.run(100)
    pa, ua = a.fields()
    pb, ub = b.fields()
    assert np.array_equal(pa, pb) and np.array_equal(ua, ub)


def test_lazy_host_tables():
    """A workload lattice (host=False) copies its host tables from the device only when read; what it then holds is
    the eager build's, bit for bit, and a solver built before any read equals one built after."""
    g = workloads.stenosed_vessel(3)
    lazy = workloads.lattice(g, 0.1)
    assert not any(k in dict.keys(lazy) for k in ("nbr", "q", "uin", "coords"))
    s0 = lbm.Solver(lazy, NU, model="regularised", order="axis-boundary-first")
    assert not any(k in dict.keys(lazy) for k in ("nbr", "q", "uin", "coords"))    # the solver read none of them
    eager = lbm.build_lattice(*_field(g, 0.1), openings=workloads.openings(g))
    for k in ("nbr", "q", "uin", "coords"):
        assert np.array_equal(lazy[k], eager[k]), k
    s1 = lbm.Solver(eager, NU, model="regularised", order="axis-boundary-first")
    for s in (s0, s1):
        workloads.configure(s, {"seed": 3, "stenosis": 0.7, "pressure": 95.0}, eager)
        s.run(50)
    p0, u0 = s0.fields()
    p1, u1 = s1.fields()
    assert np.array_equal(p0, p1) and np.array_equal(u0, u1)


def _field(g, dx):
    from cerebrosim_b200 import vessel
    phi, origin = vessel.sdf_grid(g, dx, host=False)
    return phi, origin, dx
