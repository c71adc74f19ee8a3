"""Row-sharded products and recurrences (edrixs_b200/shard.py) on world-size-2 gloo ranks on
the CPU: the reference's row partition (src/utils.f90:80-112), the exchange of x before each
product (src/spmv.f90:1-71), and the sharded Lanczos (src/lanczos.f90:210-303) and MINRES
(src/linsys.f90:3-128) recurrences with all-reduced dots.  The local product of a rank is
the oracle's CSR product of its rows (no GPU here; on GPUs it is libedx's SpMM, see
shard.csr_block_product).  Results must equal the one-rank oracle recurrences."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _problem():
    from edrixs_b200 import siam
    from oracle import pyoracle as orc
    m = siam.make_siam(4, 5, 3)
    rt = siam.text_roundtrip
    hop, coul = rt(siam.nonzero_terms(m.emat_n), 2), rt(siam.nonzero_terms(m.umat_n), 4)
    fn = orc.fock_full_N(m.nv, 6)
    H = orc.build_csr("ham_n", fn, hop, coul, num_val_orbs=m.nv, num_core_orbs=6)
    A = orc.build_csr("ham_n", fn, hop, coul, num_val_orbs=m.nv, num_core_orbs=6, ham_sign=-1.0,
                      omega=complex(35.0, 0.6))
    rng = np.random.default_rng(4)
    V = rng.normal(size=(H.nrows, 3)) + 1j * rng.normal(size=(H.nrows, 3))
    return H, A, V


def _rows_product(csr, r0, r1):
    """y_local = csr[r0:r1, :] x_full on the CPU (oracle rows), as torch."""
    import scipy.sparse as sp
    import torch
    from oracle import pyoracle as orc
    rp = csr.row_ptr[r0:r1 + 1] - csr.row_ptr[r0]
    blk = orc.CSR(rp, csr.col[csr.row_ptr[r0]:csr.row_ptr[r1]], csr.val[csr.row_ptr[r0]:csr.row_ptr[r1]], csr.ncols)
    M = sp.csr_matrix((blk.val, blk.col, blk.row_ptr), shape=(r1 - r0, csr.ncols))
    return lambda x: torch.from_numpy(M @ x.numpy())


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank))
    import torch
    from edrixs_b200 import dist, shard
    dist.init_from_env(backend="gloo", timeout_s=60)
    H, A, V = _problem()
    blocks = shard.partition_rows(H.nrows, world)
    r0, r1 = blocks[rank]
    opH = shard.RowSharded(_rows_product(H, r0, r1), H.nrows)
    a, b, nrm, neff = shard.sharded_krylov(opH, torch.from_numpy(V[r0:r1]), 25)
    opA = shard.RowSharded(_rows_product(A, r0, r1), A.nrows)
    x, it, res = shard.sharded_minres(opA, torch.from_numpy(V[r0:r1, 0]), 1e-10, 500)
    full = opA.gather(x.reshape(-1, 1))
    q.put((rank, (r0, r1), a.numpy(), b.numpy(), nrm.numpy(), neff.numpy(), full.numpy().ravel(), it, res))
    dist.finalize()


def test_partition_matches_the_reference():
    from edrixs_b200 import shard
    assert shard.partition_rows(10, 3) == [(0, 3), (3, 6), (6, 10)]
    assert shard.partition_rows(7, 1) == [(0, 7)]
    with pytest.raises(ValueError):
        shard.partition_rows(2, 3)


def test_sharded_krylov_and_minres_gloo_world2():
    from oracle import pyoracle as orc
    H, A, V = _problem()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    outs = sorted([q.get(timeout=240) for _ in range(2)], key=lambda t: t[0])
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    (_, blk0, a0, b0, n0, e0, x0, it0, r0_), (_, blk1, a1, b1, n1, e1, x1, it1, r1_) = outs
    assert blk0 == (0, H.nrows // 2) and blk1 == (H.nrows // 2, H.nrows)
    # every rank holds the same scalars
    assert np.array_equal(a0, a1) and np.array_equal(b0, b1) and np.array_equal(e0, e1) and it0 == it1
    for j in range(3):
        a_ref, b_ref, nrm_ref, neff_ref = orc.build_krylov(H, V[:, j], 25)
        assert e0[j] == neff_ref
        assert np.abs(a0[j, :neff_ref] - a_ref).max() <= 1e-10 * np.abs(a_ref).max()
        assert np.abs(b0[j, :neff_ref] - b_ref).max() <= 1e-10 * np.abs(b_ref).max()
        assert abs(n0[j] - nrm_ref) <= 1e-12 * nrm_ref
    x_ref, it_ref, res_ref = orc.minres(A, V[:, 0], 1e-10, 500)
    assert abs(it0 - it_ref) <= 2
    assert np.linalg.norm(x0 - x_ref) <= 1e-8 * np.linalg.norm(x_ref)
    assert np.array_equal(x0, x1)
