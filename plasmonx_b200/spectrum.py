"""One spectrum over several GPUs: frequency blocks per rank, results gathered
to rank 0.

The reference's three per-frequency loops (src/solvers/algorithm_module.f90:
227, 368, 438) carry no data from one frequency to the next, so a spectrum
splits into independent blocks.  Each rank (one process per GPU) holds its own
resident geometry (T or the tensor-core operand, the conductance CSR) and the
Krylov state of its block, solves the block, and the F x 20 results rows (plus
the per-frequency status and step counts, and optionally the polarizability
tensors) are gathered to rank 0 -- the only collective on the data path, a few
kilobytes per spectrum.

Partition: frequencies are dealt round-robin (rank r takes r, r + N, ...), so
every block samples the whole window: the frequencies near a plasmon
resonance, which need the most Arnoldi steps, are shared out instead of
landing on one rank.  Blocks differ in size by at most one frequency.

    from plasmonx_b200.spectrum import partition, solve_partitioned
    out = solve_partitioned(solver, prob.freqs, prob.alpha_w, pg, precision='mixed_bf16x3')
    # rank 0: out['results'] is (F, 20) in grid order; other ranks: their block only
"""
import numpy as np


def partition(n_freq, world):
    """Frequency indices of every rank: a list of `world` sorted index arrays that
    together hold 0 .. n_freq-1 exactly once."""
    if world < 1:
        raise ValueError('world size must be positive')
    return [np.arange(r, n_freq, world, dtype=np.int64) for r in range(world)]


def _gather_rows(pg, block, idx_all, rows_shape, device):
    """Rank 0 receives every rank's rows and places them at their frequency
    indices; returns the full array there and None elsewhere."""
    import torch
    rank, world = pg.get_rank(), pg.get_world_size()
    width = max(len(i) for i in idx_all)
    pad = np.zeros((width,) + rows_shape, dtype=np.float64)
    pad[:len(block)] = block
    t = torch.from_numpy(pad).to(device)
    bufs = [torch.empty_like(t) for _ in range(world)] if rank == 0 else None
    pg.gather(t, gather_list=bufs, dst=0)
    if rank != 0:
        return None
    n_freq = sum(len(i) for i in idx_all)
    full = np.zeros((n_freq,) + rows_shape, dtype=np.float64)
    for r, idx in enumerate(idx_all):
        full[idx] = bufs[r].cpu().numpy()[:len(idx)]
    return full


def solve_partitioned(solver, freqs, alpha_w, pg, device='cpu', **solve_kw):
    """Solves this rank's block of the spectrum and gathers the results.

    solver    a Solver (or any object with set_frequencies / solve) whose
              geometry is resident on this rank's device
    freqs     the whole grid (a.u.); alpha_w the whole (n_types, F) table or None
    pg        torch.distributed (initialised), or None for one rank
    device    where the gather tensors live: 'cuda:<local>' under NCCL, 'cpu' under gloo
    Returns a dict: 'results' (F, 20), 'status' (F,), 'steps' (F, 3), 'polar'
    (F, 3, 3) complex on rank 0 (None elsewhere); 'block' the rank's indices;
    'local' the rank's own solve output; 'device_ms' its device time.
    """
    rank = 0 if pg is None else pg.get_rank()
    world = 1 if pg is None else pg.get_world_size()
    idx_all = partition(len(freqs), world)
    idx = idx_all[rank]
    aw = None if alpha_w is None else np.asarray(alpha_w)[:, idx]
    solver.set_frequencies(np.asarray(freqs)[idx], aw)
    out = solver.solve(**solve_kw)
    res = {'block': idx, 'local': out, 'device_ms': float(out.get('device_ms', 0.0))}
    polar = np.asarray(out['polar'], dtype=np.complex128)
    if pg is None:
        res.update(results=out['results'], status=np.asarray(out['status']), steps=np.asarray(out['steps']),
                   polar=polar)
        return res
    cols = np.concatenate([out['results'], np.asarray(out['status'], np.float64)[:, None],
                           np.asarray(out['steps'], np.float64).reshape(len(idx), -1),
                           polar.reshape(len(idx), 9).view(np.float64)], axis=1)
    full = _gather_rows(pg, cols, idx_all, (cols.shape[1],), device)
    if full is None:
        res.update(results=None, status=None, steps=None, polar=None)
    else:
        res.update(results=full[:, :20], status=full[:, 20].astype(np.int32),
                   steps=full[:, 21:24].astype(np.int32),
                   polar=np.ascontiguousarray(full[:, 24:42]).view(np.complex128).reshape(-1, 3, 3))
    return res
