"""Grid checkpoints: save a solver's current grid to a file and restore it.

The reference has no checkpoint format; this one is defined here.  A file is

    8 bytes   magic b"LTLCKPT1"
    4 bytes   header length L (little-endian uint32)
    L bytes   UTF-8 JSON header: n (columns), rows, radius, rule
              (centre-excluded smin, smax, bmin, bmax), generation,
              words_per_row, payload_sha256, and any caller metadata under "meta"
    payload   the grid in the PACK coding: `rows` rows of words_per_row =
              ceil(n/64) little-endian uint64, cell (i, j) = bit j % 64 of word
              j / 64, bits past n zero (the layout of ltl_pack_device)

so a 32768^2 grid takes 128 MiB instead of 1 GiB.  `rows` equals n for the
square tori of ltl_create and differs for the row strips of ltl_create_rect; a
header without it (older files) means rows = n.  On the device path the grid
is packed by ltl_pack_device before the download and unpacked by
ltl_unpack_device after the upload, so only the packed bytes cross PCIe.
`read` checks the magic, the sizes and the payload's SHA-256; `load` refuses a
solver whose n, rows, radius or rule differ from the header's.
"""
import ctypes
import hashlib
import json
import struct

import numpy as np

MAGIC = b"LTLCKPT1"


def words_per_row(n):
    return (n + 63) // 64


def pack_host(grid):
    """uint8 rows x n (0/1) -> uint64 rows in the PACK coding (numpy, host side)."""
    g = np.ascontiguousarray(grid, dtype=np.uint8)
    n = g.shape[1]
    wpr = words_per_row(n)
    padded = np.zeros((g.shape[0], wpr * 64), dtype=np.uint8)
    padded[:, :n] = g & 1
    bits = np.packbits(padded.reshape(g.shape[0], wpr, 64), axis=2, bitorder="little")  # 8 bytes per word
    return bits.reshape(g.shape[0], wpr * 8).view("<u8")


def unpack_host(words, n):
    """PACK-coded uint64 rows -> uint8 rows x n."""
    w = np.ascontiguousarray(words, dtype="<u8")
    b = np.unpackbits(w.view(np.uint8).reshape(w.shape[0], -1), axis=1, bitorder="little")
    return b[:, :n].astype(np.uint8)


def _header(n, radius, rule, generation, payload, meta, rows):
    return {"n": int(n), "rows": int(rows), "radius": int(radius), "rule": [int(x) for x in rule],
            "generation": int(generation), "words_per_row": words_per_row(n),
            "payload_sha256": hashlib.sha256(payload).hexdigest(), "meta": meta or {}}


def write(path, words, n, radius, rule, generation=0, meta=None, rows=None):
    rows = n if rows is None else int(rows)
    payload = np.ascontiguousarray(words, dtype="<u8").tobytes()
    if len(payload) != rows * words_per_row(n) * 8:
        raise ValueError("payload size does not match rows x n")
    head = json.dumps(_header(n, radius, rule, generation, payload, meta, rows), sort_keys=True).encode()
    with open(path, "wb") as f:
        f.write(MAGIC)
        f.write(struct.pack("<I", len(head)))
        f.write(head)
        f.write(payload)


def read(path):
    """-> (header dict, uint64 words of shape (rows, words_per_row)).  Raises ValueError
    on a bad magic, a truncated file or a checksum mismatch.  The header always
    carries "rows" (n for files written without it)."""
    with open(path, "rb") as f:
        if f.read(8) != MAGIC:
            raise ValueError(f"{path}: not a grid checkpoint")
        (hl,) = struct.unpack("<I", f.read(4))
        head = json.loads(f.read(hl).decode())
        payload = f.read()
    n, wpr = head["n"], head["words_per_row"]
    rows = head.setdefault("rows", n)
    if wpr != words_per_row(n) or len(payload) != rows * wpr * 8:
        raise ValueError(f"{path}: truncated or inconsistent checkpoint")
    if hashlib.sha256(payload).hexdigest() != head["payload_sha256"]:
        raise ValueError(f"{path}: checksum mismatch")
    return head, np.frombuffer(payload, dtype="<u8").reshape(rows, wpr).copy()


def save(path, solver, generation=0, meta=None):
    """Write `solver`'s current grid (rows x n; rows = n unless the solver is a
    rectangular strip).  Packs on the device (ltl_pack_device) and downloads the
    packed words only."""
    import torch
    from . import ltl
    n = solver.n
    rows = getattr(solver, "rows", n)
    wpr = words_per_row(n)
    dev = torch.device("cuda", solver.device)
    cells = torch.empty((rows, n), dtype=torch.uint8, device=dev)
    words = torch.empty((rows, wpr), dtype=torch.int64, device=dev)
    torch.cuda.synchronize(dev)
    solver.download_device(cells.data_ptr(), n)
    solver.synchronize()
    ltl.check(ltl.lib().ltl_pack_device(ctypes.c_void_p(cells.data_ptr()), n, rows, n,
                                        ctypes.c_void_p(words.data_ptr()), wpr * 8, None))
    torch.cuda.synchronize(dev)
    host = words.cpu().numpy().view("<u8")
    write(path, host, n, solver.radius, solver.rule, generation, meta, rows=rows)


def check_compatible(head, solver):
    """Raise ValueError unless `solver` has the checkpoint's shape, radius and rule:
    restoring a grid into a solver with another rule would step it under that rule."""
    want = (head["n"], head["rows"], head["radius"], tuple(head["rule"]))
    have = (solver.n, getattr(solver, "rows", solver.n), solver.radius, tuple(solver.rule))
    for name, a, b in zip(("n", "rows", "radius", "rule"), want, have):
        if a != b:
            raise ValueError(f"checkpoint holds {name}={a}, solver has {name}={b}")


def load(path, solver=None, variant=None, device=0):
    """Restore a checkpoint into `solver` (same n, rows, radius and rule, else
    ValueError), or into a new CUDASolver built from the header (a rectangular
    one for a strip).  Returns (solver, header)."""
    head, host = read(path)
    n, rows = head["n"], head["rows"]
    if solver is not None:
        check_compatible(head, solver)
    import torch
    from . import ltl
    if solver is None:
        kw = {} if variant is None else {"variant": variant}
        if rows != n:
            kw["rows"] = rows
        solver = ltl.CUDASolver(n, head["radius"], tuple(head["rule"]), device=device, **kw)
    dev = torch.device("cuda", solver.device)
    words = torch.from_numpy(host.view(np.int64)).to(dev)
    cells = torch.empty((rows, n), dtype=torch.uint8, device=dev)
    ltl.check(ltl.lib().ltl_unpack_device(ctypes.c_void_p(words.data_ptr()), head["words_per_row"] * 8, rows, n,
                                          ctypes.c_void_p(cells.data_ptr()), n, None))
    torch.cuda.synchronize(dev)
    solver.upload_device(cells.data_ptr(), n)
    solver.synchronize()
    return solver, head
