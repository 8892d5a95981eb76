"""The reference's Frechet-row file (SurfTime::frechet_matrix,
src/SWD/SurfaceWave.cpp:596-603 and 641-659): per rank file, a header of
int32 m (data count) and int32 n = (nx-2)(ny-2)(nz-1), then one record per
(pair, receiver) row: int32 row id, int32 nnz, int32 idx[nnz] (ascending),
float32 val[nnz].  Written here from the device CSR rows
(swdk_frechet_csr_device) so the LSMR side reads it unchanged."""
import numpy as np


def write_frechet(path, m, n, row_ids, rowptr, indices, values):
    row_ids = np.asarray(row_ids, np.int32)
    rowptr = np.asarray(rowptr, np.int64)
    indices = np.asarray(indices, np.int32)
    values = np.asarray(values, np.float32)
    with open(path, "wb") as f:
        f.write(np.array([m, n], np.int32).tobytes())
        for r, rid in enumerate(row_ids):
            a, b = int(rowptr[r]), int(rowptr[r + 1])
            f.write(np.array([rid, b - a], np.int32).tobytes())
            f.write(indices[a:b].tobytes())
            f.write(values[a:b].tobytes())


def write_frechet_device(path, m, n, rowptr, indices, values, row_id0=0, row_ids=None, stream=None):
    """The same file from CSR rows on the device (torch tensors): the record
    stream is built by swdk_frechet_records_device on the GPU, copied to the
    host in one piece and written with one write.  `stream` is the CUDA stream
    handle the rows were made on (None: torch's current stream)."""
    import ctypes as C

    import torch
    from .engine import _p, lib
    L = lib()
    fn = L.swdk_frechet_records_device
    vp = C.c_void_p
    fn.argtypes = [C.c_int64, C.c_int32, C.c_int32, vp, C.c_int32, vp, vp, vp, C.c_int64, vp, C.c_int64, vp]
    nrow = rowptr.shape[0] - 1
    nnz = int(rowptr[-1].item()) if nrow > 0 else 0
    words = 2 + 2 * nrow + 2 * nnz
    out = torch.empty(words, dtype=torch.int32, device=rowptr.device)
    sp = stream if stream is not None else torch.cuda.current_stream(rowptr.device).cuda_stream
    torch.cuda.synchronize(rowptr.device)  # `out` was allocated on torch's stream
    rc = fn(nrow, m, n, _p(row_ids), int(row_id0), _p(rowptr), _p(indices), _p(values), nnz, _p(out), words,
            C.c_void_p(sp))
    if rc != 0:
        raise RuntimeError(f"swdk_frechet_records_device failed ({rc})")
    torch.cuda.synchronize(rowptr.device)  # the records were built on `sp`
    host = out.cpu()
    with open(path, "wb") as f:
        f.write(host.numpy().tobytes())


def read_frechet(path):
    """-> (m, n, [(row id, idx int32[], val float32[]), ...])"""
    raw = open(path, "rb").read()
    m, n = np.frombuffer(raw, np.int32, 2, 0)
    pos, rows = 8, []
    while pos < len(raw):
        rid, nnz = np.frombuffer(raw, np.int32, 2, pos)
        pos += 8
        idx = np.frombuffer(raw, np.int32, nnz, pos)
        pos += 4 * nnz
        val = np.frombuffer(raw, np.float32, nnz, pos)
        pos += 4 * nnz
        rows.append((int(rid), idx.copy(), val.copy()))
    return int(m), int(n), rows


def merge_frechet(parts, outfile, remove=True):
    """The reference's merge_csr_files (src/shared/csr_matrix.cpp:205-242):
    per-rank row files outfile.0, outfile.1, ... (each with its own m, n
    header) concatenated into one file with the first header."""
    import os
    with open(outfile, "wb") as out:
        for i, part in enumerate(parts):
            with open(part, "rb") as f:
                head = f.read(8)
                if i == 0:
                    out.write(head)
                out.write(f.read())
            if remove:
                os.remove(part)
