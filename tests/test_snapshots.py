"""Snapshot files in H5Saver's layout (simulation/set_simulator.py:126-318)
and restarts.

No HDF5 library is importable in this image (h5py absent), so H5Saver runs on
janc_b200.h5lite here.  CPU: h5lite round trips (groups, attributes, gzip
and contiguous datasets, appends across reopenings, deletions, groups larger
than one symbol-table node) and byte-level checks of the structures the HDF5
file format specification fixes (superblock version 0, end-of-file address,
version-1 object headers, the local heap's leading empty name, names sorted
across symbol-table nodes and B-tree keys); the reader on hand-assembled
structures its writer does not produce but h5py files contain (object header
continuations, attribute messages 2 and 3, dataspace 2, compact layout,
multi-chunk shuffle + deflate datasets, version-2 object headers with link
messages); H5Saver's save / parallel layout / collect / load_state.  The
files are not opened by libhdf5 here: their compatibility with it is
unpinned.
GPU: Simulator.run writes the snapshots; a restart from a middle snapshot
reproduces the uninterrupted run bit for bit; load / load_all primitives.
"""
import struct

import numpy as np
import pytest

from janc_b200 import h5lite


def test_h5lite_roundtrip(tmp_path):
    p = tmp_path / "a.h5"
    f = h5lite.File(p, "w")
    g = f.create_group("save_step0")
    g.attrs["time"] = np.float64(0.25)
    g.attrs["step"] = np.int64(7)
    g.attrs["vec"] = np.arange(3, dtype=np.float32)
    g.attrs["name"] = "detonation"
    rng = np.random.default_rng(0)
    u = rng.standard_normal((12, 17, 9))
    g.create_dataset("u", data=u, compression="gzip")
    g.create_dataset("aux", data=u[:2].astype(np.float32))
    g.create_dataset("ids", data=np.arange(10, dtype=np.int64))
    g.create_dataset("scalar", data=np.float64(3.5), compression="gzip")
    g.create_dataset("empty", data=np.zeros((0, 4)))
    f.close()
    f = h5lite.File(p, "r")
    g = f["save_step0"]
    assert g.attrs["time"] == 0.25 and g.attrs["step"] == 7 and g.attrs["name"] == b"detonation"
    assert np.array_equal(g.attrs["vec"], np.arange(3, dtype=np.float32))
    assert np.array_equal(np.asarray(g["u"]), u) and g["u"].shape == (12, 17, 9)
    assert np.array_equal(np.asarray(g["aux"]), u[:2].astype(np.float32))
    assert np.array_equal(g["ids"][2:5], [2, 3, 4])
    assert np.asarray(g["scalar"]) == 3.5 and g["empty"].shape == (0, 4)
    assert sorted(g.keys()) == ["aux", "empty", "ids", "scalar", "u"]
    f.close()


def test_h5lite_append_delete_and_many_groups(tmp_path):
    p = tmp_path / "b.h5"
    for k in range(150):  # more than one symbol-table node (64 links) per group
        f = h5lite.File(p, "a")
        grp = f.create_group(f"save_step{k}")
        grp.attrs["time"] = 0.1 * k
        grp.create_dataset("u", data=np.full((2, 3), float(k)), compression="gzip" if k % 2 else None)
        f.close()
    f = h5lite.File(p, "a")
    del f["save_step3"]
    f.create_group("save_step3").create_dataset("u", data=np.full((2, 3), -1.0))
    f.close()
    f = h5lite.File(p, "r")
    assert len(f.keys()) == 150
    for k in (0, 1, 63, 64, 65, 99, 149):
        assert np.all(np.asarray(f[f"save_step{k}"]["u"]) == float(k))
        assert f[f"save_step{k}"].attrs["time"] == 0.1 * k
    assert np.all(np.asarray(f["save_step3"]["u"]) == -1.0) and "time" not in f["save_step3"].attrs
    f.close()


def test_h5lite_structures_follow_the_format(tmp_path):
    p = tmp_path / "c.h5"
    f = h5lite.File(p, "w")
    names = [f"save_step{k}" for k in range(70)]
    for n in names:
        f.create_group(n)
    f.close()
    b = p.read_bytes()
    assert b[:8] == b"\x89HDF\r\n\x1a\n" and b[8] == 0 and b[13] == 8 and b[14] == 8
    leaf_k, int_k = struct.unpack_from("<HH", b, 16)
    eof = struct.unpack_from("<Q", b, 40)[0]
    assert eof == len(b) and eof % 8 == 0
    root, cache, _, bt, heap = struct.unpack_from("<QII QQ".replace(" ", ""), b, 64)
    assert cache == 1 and b[root] == 1  # cached symbol table, version-1 object header
    nmsg, _, size = struct.unpack_from("<HII", b, root + 2)
    t, n = struct.unpack_from("<HH", b, root + 16)
    assert (nmsg, t, n) == (1, 0x11, 16) and struct.unpack_from("<QQ", b, root + 24) == (bt, heap)
    assert b[heap:heap + 4] == b"HEAP"
    dsize, free, daddr = struct.unpack_from("<QQQ", b, heap + 8)
    assert free == h5lite.FREE_NULL and b[daddr:daddr + 8] == b"\0" * 8
    assert b[bt:bt + 6] == b"TREE\x00\x00"
    nsn = struct.unpack_from("<H", b, bt + 6)[0]
    assert nsn == -(-70 // (2 * leaf_k))
    keys = [struct.unpack_from("<Q", b, bt + 24 + 16 * i)[0] for i in range(nsn + 1)]
    kids = [struct.unpack_from("<Q", b, bt + 32 + 16 * i)[0] for i in range(nsn)]

    def name(off):
        return b[daddr + off:b.index(b"\0", daddr + off)]
    got = []
    for i, s in enumerate(kids):
        assert b[s:s + 5] == b"SNOD\x01"
        cnt = struct.unpack_from("<H", b, s + 6)[0]
        ns = [name(struct.unpack_from("<Q", b, s + 8 + 40 * j)[0]) for j in range(cnt)]
        assert ns == sorted(ns) and name(keys[i + 1]) == ns[-1] and (i == 0 or name(keys[i]) < ns[0])
        got += ns
    assert keys[0] == 0 and got == sorted(n.encode() for n in names)


def test_h5saver_layout_and_collect(tmp_path):
    from janc_b200.janc.simulation.set_simulator import H5Saver
    p = tmp_path / "s.h5"
    s = H5Saver(p, "2D")
    U = np.arange(2 * 8 * 3, dtype=np.float64).reshape(2, 8, 3)
    aux = np.ones((2, 8, 3))
    s.save(0, 0.0, 0, u=U, aux=aux)
    s.save(1, 1e-6, 5, u=U + 1, aux=aux)
    s.save(1, 2e-6, 6, u=U + 2, aux=aux)  # an existing group is replaced
    for d in range(2):  # the layout parallel_save writes, one group per slab
        s._write(f"save_step2_device{d}", 3e-6, 9, {"u": U[:, 4 * d:4 * d + 4], "aux": aux[:, 4 * d:4 * d + 4]})
    s.collect()
    assert sorted(s.list_snapshots()) == ["save_step0", "save_step1", "save_step2", "save_step2_device0",
                                          "save_step2_device1"]
    U1, a1, t1, st1 = s.load_state("save_step1")
    assert np.array_equal(U1, U + 2) and (t1, st1) == (2e-6, 6)
    U2, a2, t2, st2 = s.load_state()
    assert np.array_equal(U2, U) and (t2, st2) == (3e-6, 9)
    s.close()
    f = h5lite.File(p, "r")
    g = f["save_step1"]
    assert sorted(g.keys()) == ["aux", "u"] and g["u"].shape == (2, 8, 3)
    assert g.attrs["time"].dtype == np.float64 and g.attrs["step"].dtype == np.int64
    f.close()


# ---------------------------------------------------------------- GPU
def _config(tmp_path, save_dt, t_end):
    from janc_b200.mechanism import DEFAULT_MECHANISM as MECH
    return {"dimension": "1D", "grid_config": {"dx": 5e-5},
            "thermo_config": {"thermo_model": "nasa7", "mechanism_directory": MECH},
            "reaction_config": {"is_detailed_chemistry": True, "mechanism_directory": MECH},
            "flux_config": {"solver_type": "flux_splitting", "interface_reconstruction": "WENO5_JS",
                            "split_method": "LF", "viscosity": "off"},
            "boundary_config": {"left_boundary": "slip_wall", "right_boundary": "zero_gradient"},
            "time_config": {"temporal_evolution_scheme": "TVD_RK3", "t_end": t_end, "CFL": 0.5},
            "computation_config": {"output_settings": {"save_dt": save_dt,
                                                       "results_path": str(tmp_path / "run.h5")}}}


def _tube(nx=400):
    """A 5:1 shock tube at 300 K (finite for the whole run; a 30 atm / 3000 K
    slab at CFL 0.5 goes non-finite within tens of steps, as the reference's
    does)."""
    from oracle import janc_oracle as jo
    from janc_b200.mechanism import DEFAULT_MECHANISM
    m = jo.load_mechanism(DEFAULT_MECHANISM)
    P = np.full((1, nx), 101325.0)
    T = np.full((1, nx), 300.0)
    P[:, :40] = 5 * 101325.0
    return jo.state_from_PTY(m, P, T, np.tile(jo.stoich_Y(m, 1.0)[:, None], (1, nx)))


@pytest.mark.gpu
def test_run_snapshots_and_bitwise_restart(tmp_path):
    from janc_b200.janc.simulation.set_simulator import H5Saver, Simulator
    U0, a0 = _tube()
    sim = Simulator(_config(tmp_path, 2e-7, 1e-6))
    U, aux, t = sim.run(U0, a0)
    assert np.isfinite(t) and np.all(np.isfinite(U))
    s = H5Saver(tmp_path / "run.h5", "1D", mode="r")
    keys = sorted(s.list_snapshots(), key=lambda k: int(k[9:]))
    times = [s.load_state(k)[2] for k in keys]
    assert keys[0] == "save_step0" and times[0] == 0.0 and len(keys) == 6
    assert all(b > a for a, b in zip(times, times[1:])) and times[-1] == t
    Ul, al, tl, stl = s.load_state()
    assert np.array_equal(Ul, U) and np.array_equal(al, aux)
    tm, prim = s.load(keys[2])
    assert set(prim) == {"density", "x-velocity", "pressure", "tempreature", "species"}
    assert prim["species"].shape == (8, 400) and np.all(prim["pressure"] > 0)
    ts, allp = s.load_all()
    assert ts.shape == (6,) and allp["density"].shape == (6, 400)
    s.close()
    # restart from snapshot 2 into a new file: the same final state, bit for bit
    Ur, ar, tr, str_ = Simulator(_config(tmp_path, 2e-7, 1e-6)).restart("save_step2")
    sim2 = Simulator(_config(tmp_path, 2e-7, 1e-6))
    sim2.results_path = str(tmp_path / "restart.h5")
    U2, a2, t2 = sim2.run(Ur, ar, t0=tr, step0=str_)
    assert t2 == t and np.array_equal(U2, U) and np.array_equal(a2, aux)
    s2 = H5Saver(tmp_path / "restart.h5", "1D", mode="r")
    assert "save_step0" not in s2.list_snapshots() and "save_step5" in s2.list_snapshots()
    s2.close()
    # a snapshot as the reference writes it (u only): aux from the temperature solve
    f = h5lite.File(tmp_path / "u_only.h5", "w")
    g = f.create_group("save_step0")
    g.attrs["time"] = 0.0
    g.attrs["step"] = 0
    g.create_dataset("u", data=U0, compression="gzip")
    f.close()
    s3 = H5Saver(tmp_path / "u_only.h5", "1D", mode="r")
    U3, a3, t3, _ = s3.load_state()
    s3.close()
    assert np.array_equal(U3, U0) and np.max(np.abs(a3[1] - a0[1]) / a0[1]) < 1e-9


def _parallel_worker(rank, size, port, out):
    import datetime
    import torch
    import torch.distributed as dist
    from janc_b200.janc.parallel.grid_partion import gather_grid
    from janc_b200.janc.simulation.set_simulator import Simulator
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=size,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import pathlib
        cfg = _config(pathlib.Path(out), 2e-7, 6e-7)
        cfg["computation_config"]["is_parallel"] = True
        sim = Simulator(cfg)
        U0, a0 = _tube()
        U, aux, t = sim.run(U0, a0)
        Ug, ag = gather_grid(U), gather_grid(aux)
        Ur, ar, tr, sr = sim.restart()
        np.savez(pathlib.Path(out) / f"p{rank}.npz", U=Ug.cpu().numpy(), aux=ag.cpu().numpy(), t=t,
                 Ur=Ur, ar=ar, tr=tr)
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_parallel_snapshots_collect_and_restart(tmp_path):
    """Slabs as two gloo ranks on one GPU: rank 0 writes save_step{k}_device{d}
    groups; restart() collects them into the global state."""
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    mp.start_processes(_parallel_worker, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn")
    for r in range(2):
        d = np.load(tmp_path / f"p{r}.npz")
        assert np.array_equal(d["Ur"], d["U"]) and np.array_equal(d["ar"], d["aux"])
        assert float(d["tr"]) == float(d["t"])
    f = h5lite.File(tmp_path / "run.h5", "r")
    keys = set(f.keys())
    assert {"save_step0_device0", "save_step0_device1", "save_step0", "save_step3"} <= keys
    assert f["save_step0_device1"]["u"].shape == (11, 200) and f["save_step0"]["u"].shape == (11, 400)
    f.close()


# ------------------------------------------------ reader paths h5py files use
def _h5_file(objs, root_addr_key="root"):
    """Assemble a file from hand-built objects: objs is an ordered list of
    (name, bytes-builder(addr_of) -> bytes); addresses are assigned in order
    after a version-0 superblock."""
    import struct as st
    addr, blobs = {}, []
    pos = 96
    for name, build in objs:
        addr[name] = pos
        size = len(build(lambda k: 0))
        pos += size + (-size % 8)
    for name, build in objs:
        b = build(lambda k: addr[k])
        blobs.append(b + b"\0" * (-len(b) % 8))
    sb = (b"\x89HDF\r\n\x1a\n" + st.pack("<8BHHI", 0, 0, 0, 0, 0, 8, 8, 0, 4, 16, 0)
          + st.pack("<QQQQ", 0, 0xFFFFFFFFFFFFFFFF, pos, 0xFFFFFFFFFFFFFFFF)
          + st.pack("<QQII", 0, addr[root_addr_key], 0, 0) + b"\0" * 16)
    return sb + b"".join(blobs)


def test_h5lite_reads_continuations_v2_v3_messages_and_chunks(tmp_path):
    """Structures h5py / libhdf5 write that h5lite's writer does not:
    a version-1 object header continued in a second block, attribute
    messages of versions 2 and 3, a version-2 dataspace, a compact layout,
    a chunked dataset of several chunks with shuffle + deflate, a
    version-2 object header with compact link messages."""
    import struct as st
    import zlib
    H = h5lite
    f64 = H._encode_dtype(np.float64)
    i32 = H._encode_dtype(np.int32)

    def msg1(t, data, fl=0):
        data = H._pad8(data)
        return st.pack("<HHB3x", t, len(data), fl) + data

    def attr_v3(name, val):
        v = np.asarray(val, dtype=np.float64)
        nm = name.encode() + b"\0"
        sp = st.pack("<BBBB", 2, 1, 0, 1) + st.pack("<Q", v.size)  # dataspace v2, simple
        return st.pack("<BBHHHB", 3, 0, len(nm), len(f64), len(sp), 0) + nm + f64 + sp + v.tobytes()

    def attr_v2(name, val):
        v = np.asarray(val, dtype=np.int32)
        nm = name.encode() + b"\0"
        sp = st.pack("<BBBB", 2, 0, 0, 0)  # scalar dataspace v2
        return st.pack("<BBHHH", 2, 0, len(nm), len(i32), len(sp)) + nm + i32 + sp + v.tobytes()

    a = np.arange(6 * 10, dtype=np.float64).reshape(6, 10) * 0.5
    chunks = {}
    for cx in (0, 4):
        for cy in (0, 4, 8):
            c = np.zeros((4, 4))
            blk = a[cx:cx + 4, cy:cy + 4]
            c[:blk.shape[0], :blk.shape[1]] = blk
            sh = np.frombuffer(c.tobytes(), np.uint8).reshape(-1, 8).T.tobytes()  # shuffle
            chunks[(cx, cy)] = zlib.compress(sh)
    keys = sorted(chunks)
    ks = 8 + 8 * 3

    def btree(A):
        body = b""
        for i, k in enumerate(keys):
            body += st.pack("<II3Q", len(chunks[k]), 0, k[0], k[1], 0) + st.pack("<Q", A(f"c{i}"))
        body += st.pack("<II3Q", 0, 0, 6, 10, 0)
        node = b"TREE" + bytes([1, 0]) + st.pack("<HQQ", len(keys), H.UNDEF, H.UNDEF) + body
        return node + b"\0" * (24 + 64 * 8 + 65 * ks - len(node))

    filt = (st.pack("<BB6x", 1, 2) + st.pack("<HHHH", 2, 8, 0, 1) + H._pad8(b"shuffle\0") + st.pack("<I4x", 8)
            + st.pack("<HHHH", 1, 8, 0, 1) + H._pad8(b"deflate\0") + st.pack("<I4x", 6))

    def ds_chunked(A):
        msgs = (msg1(1, H._space_msg((6, 10))) + msg1(3, f64, 1)
                + msg1(8, st.pack("<BBBQ3I", 3, 2, 3, A("bt"), 4, 4, 8)) + msg1(11, filt))
        return st.pack("<BBHII4x", 1, 0, 4, 1, len(msgs)) + msgs

    small = np.array([1.5, -2.0, 7.25])

    def ds_compact(A):
        lay = st.pack("<BBH", 3, 0, small.nbytes) + small.tobytes()
        msgs = msg1(1, st.pack("<BBBB", 2, 1, 0, 1) + st.pack("<Q", 3)) + msg1(3, f64, 1) + msg1(8, lay)
        return st.pack("<BBHII4x", 1, 0, 3, 1, len(msgs)) + msgs

    def grp(A):  # version-1 header: link table in a continuation block
        cont = msg1(16, st.pack("<QQ", A("cont"), len(grp_cont(A))))
        msgs = msg1(12, attr_v3("time", [2.5e-6])) + cont
        return st.pack("<BBHII4x", 1, 0, 3, 1, len(msgs)) + msgs

    def grp_cont(A):
        return msg1(12, attr_v2("step", 42)) + msg1(17, st.pack("<QQ", A("gbt"), A("gheap")))

    names = [b"chunked", b"compact"]
    heap_data = b"\0" * 8 + H._pad8(names[0] + b"\0") + H._pad8(names[1] + b"\0")
    offs = [8, 8 + len(H._pad8(names[0] + b"\0"))]

    def gheap(A):
        return b"HEAP" + bytes(4) + st.pack("<QQQ", len(heap_data), H.FREE_NULL, A("gheapdata"))

    def gsnod(A):
        ent = b"".join(st.pack("<QQII16x", o, A(n), 0, 0) for o, n in zip(offs, ("ds1", "ds2")))
        return b"SNOD" + bytes([1, 0]) + st.pack("<H", 2) + ent + b"\0" * (40 * 6)

    def gbt(A):
        node = (b"TREE" + bytes([0, 0]) + st.pack("<HQQ", 1, H.UNDEF, H.UNDEF)
                + st.pack("<QQQ", 0, A("gsnod"), offs[1]))
        return node + b"\0" * (24 + 32 * 8 + 33 * 8 - len(node))

    def root(A):  # version-2 object header with one compact hard link
        link = bytes([1, 0x00]) + bytes([len(b"save_step7")]) + b"save_step7" + st.pack("<Q", A("grp"))
        body = bytes([6]) + st.pack("<H", len(link)) + bytes([0]) + link
        return b"OHDR" + bytes([2, 0]) + bytes([len(body)]) + body + b"\0\0\0\0"

    objs = [("root", root), ("grp", grp), ("cont", grp_cont), ("gbt", gbt), ("gsnod", gsnod), ("gheap", gheap),
            ("gheapdata", lambda A: heap_data), ("ds1", ds_chunked), ("ds2", ds_compact), ("bt", btree)]
    objs += [(f"c{i}", (lambda k: lambda A: chunks[k])(k)) for i, k in enumerate(keys)]
    p = tmp_path / "handmade.h5"
    p.write_bytes(_h5_file(objs))
    f = h5lite.File(p, "r")
    assert list(f.keys()) == ["save_step7"]
    g = f["save_step7"]
    assert g.attrs["time"] == 2.5e-6 and g.attrs["step"] == 42
    assert sorted(g.keys()) == ["chunked", "compact"]
    assert np.array_equal(np.asarray(g["chunked"]), a)
    assert np.array_equal(np.asarray(g["compact"]), small)
    f.close()
