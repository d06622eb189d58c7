"""The production streaming pipeline (bench.py --workload stream; config 5's
1e8 C2H6-like explosions), checked chunk by chunk.

Per chunk, on a compute stream: Philox geometries on the device, then the
integration (ce_run_device, the fixed-molecule entry point) replayed from a CUDA
graph captured once per buffer slot; on a side stream: the chunk's momenta / KER
/ steps / status copied into a two-slot pinned host ring that the host reads
while the next chunk computes. This replaces the reference's production loop
(examples/generate_dataset.cpp:159-240). Every chunk read from the ring must
equal, bit for bit, an eager ce_run_device of the same geometries, and the first
chunk must match the FP64 oracle on a subset within the tight-point tolerance.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle_lib as ol
from pkg_loader import load_submodule

pytestmark = pytest.mark.gpu

TIGHT_MAX = 1e-5


def test_graph_replayed_chunks_in_the_pinned_ring_equal_ce_run_device(ce, wl):
    torch = pytest.importorskip("torch")
    cl = load_submodule("closure")
    sp = load_submodule("sampling")
    lib = ce.load_library()
    dev = torch.device("cuda", 0)
    mol = wl.C2H6_LIKE
    Cn, nchunks, seed = 1 << 16, 4, 424242
    cfg = ce.RunConfig(rtol=wl.TIGHT[0], atol=wl.TIGHT[1], pe_stop_fraction=wl.TIGHT[2], precision_mode=0)
    eng = ce.Engine(0)
    try:
        eng.set_molecule(mol.masses_me, mol.charge_array)
        slots = []
        for _ in range(2):
            b = cl.sample_molecule_device(mol, Cn, seed, first_sim=0)
            d = {"batch": b, "cb": b.c(),
                 "momenta": torch.empty((Cn, 10, 3), dtype=torch.float32, device=dev),
                 "ker": torch.empty(Cn, dtype=torch.float64, device=dev),
                 "steps": torch.empty(Cn, dtype=torch.int32, device=dev),
                 "status": torch.empty(Cn, dtype=torch.uint8, device=dev)}
            d["out"] = ce.CeOutputs(d["momenta"].data_ptr(), d["ker"].data_ptr(), d["steps"].data_ptr(),
                                    d["status"].data_ptr())
            d["host"] = {k: torch.empty(d[k].shape, dtype=d[k].dtype, pin_memory=True)
                         for k in ("momenta", "ker", "steps", "status")}
            slots.append(d)
        compute, side = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)
        cs = compute.cuda_stream
        graphs = []
        for d in slots:  # eager call first (sets the kernel attributes), then the capture
            eng.run_device(Cn, d["batch"].pos.data_ptr(), cfg, d["out"], cs)
            torch.cuda.synchronize()
            eng.graph_begin(cs)
            eng.run_device(Cn, d["batch"].pos.data_ptr(), cfg, d["out"], cs)
            graphs.append(eng.graph_end(cs))
        bcfg = sp.ball_config(mol, seed)
        done = [torch.cuda.Event() for _ in range(2)]
        copied = [torch.cuda.Event() for _ in range(2)]
        got = []

        def consume(i):
            d = slots[i % 2]
            copied[i % 2].synchronize()
            got.append({k: v.clone() for k, v in d["host"].items()})

        for i in range(nchunks):
            d = slots[i % 2]
            if i >= 2:
                compute.wait_event(copied[i % 2])
            assert lib.ce_sample_ball_device(10, i * Cn, Cn, C.byref(bcfg), C.c_void_p(d["batch"].pos.data_ptr()),
                                             None, C.c_void_p(cs)) == 0
            graphs[i % 2].launch(cs)
            done[i % 2].record(compute)
            side.wait_event(done[i % 2])
            with torch.cuda.stream(side):
                for k in ("momenta", "ker", "steps", "status"):
                    d["host"][k].copy_(d[k], non_blocking=True)
            copied[i % 2].record(side)
            if i >= 1:
                consume(i - 1)
        consume(nchunks - 1)
        torch.cuda.synchronize()
        for g in graphs:
            g.close()

        # The same geometries through the same entry point, eagerly.
        pos = torch.empty((Cn, 10, 3), dtype=torch.float32, device=dev)
        ref = {"momenta": torch.empty((Cn, 10, 3), dtype=torch.float32, device=dev),
               "ker": torch.empty(Cn, dtype=torch.float64, device=dev),
               "steps": torch.empty(Cn, dtype=torch.int32, device=dev),
               "status": torch.empty(Cn, dtype=torch.uint8, device=dev)}
        rout = ce.CeOutputs(ref["momenta"].data_ptr(), ref["ker"].data_ptr(), ref["steps"].data_ptr(),
                            ref["status"].data_ptr())
        s0 = torch.cuda.current_stream().cuda_stream
        for i, g in enumerate(got):
            assert lib.ce_sample_ball_device(10, i * Cn, Cn, C.byref(bcfg), C.c_void_p(pos.data_ptr()), None,
                                             C.c_void_p(s0)) == 0
            eng.run_device(Cn, pos.data_ptr(), cfg, rout, s0)
            torch.cuda.synchronize()
            assert (g["status"].numpy() == 0).all(), i
            for k in ("momenta", "ker", "steps", "status"):
                np.testing.assert_array_equal(g[k].numpy(), ref[k].cpu().numpy(), err_msg=f"chunk {i} {k}")
            if i == 0:
                sub = np.arange(0, Cn, Cn // 64)
                x = pos.cpu().numpy()[sub].astype(np.float64)
                o = ol.run_batch(x, mol.masses_me, mol.charge_array, bits=64, rtol=1e-10, atol=1e-16,
                                 pe_stop=1e-11)
                err = ol.config_norm_error(g["momenta"].numpy()[sub], o["momenta"])
                assert err.max() <= TIGHT_MAX, err.max()
    finally:
        eng.close()
