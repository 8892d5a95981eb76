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
