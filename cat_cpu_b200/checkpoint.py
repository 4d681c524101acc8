"""Grid checkpoints: save a solver's current grid to a file and restore it.

The reference has no checkpoint format; this one is defined here.  A file is

    8 bytes   magic b"LTLCKPT1"
    4 bytes   header length L (little-endian uint32)
    L bytes   UTF-8 JSON header: n, radius, rule (centre-excluded smin, smax,
              bmin, bmax), generation, words_per_row, payload_sha256, and any
              caller metadata under "meta"
    payload   the grid in the PACK coding: n rows of words_per_row = ceil(n/64)
              little-endian uint64, cell (i, j) = bit j % 64 of word j / 64, bits
              past n zero (the layout of ltl_pack_device)

so a 32768^2 grid takes 128 MiB instead of 1 GiB.  On the device path the grid
is packed by ltl_pack_device before the download and unpacked by
ltl_unpack_device after the upload, so only the packed bytes cross PCIe.
`read` checks the magic, the sizes and the payload's SHA-256.
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


def _header(n, radius, rule, generation, payload, meta):
    return {"n": int(n), "radius": int(radius), "rule": [int(x) for x in rule], "generation": int(generation),
            "words_per_row": words_per_row(n), "payload_sha256": hashlib.sha256(payload).hexdigest(),
            "meta": meta or {}}


def write(path, words, n, radius, rule, generation=0, meta=None):
    payload = np.ascontiguousarray(words, dtype="<u8").tobytes()
    if len(payload) != n * words_per_row(n) * 8:
        raise ValueError("payload size does not match n")
    head = json.dumps(_header(n, radius, rule, generation, payload, meta), sort_keys=True).encode()
    with open(path, "wb") as f:
        f.write(MAGIC)
        f.write(struct.pack("<I", len(head)))
        f.write(head)
        f.write(payload)


def read(path):
    """-> (header dict, uint64 words of shape (n, words_per_row)).  Raises ValueError on
    a bad magic, a truncated file or a checksum mismatch."""
    with open(path, "rb") as f:
        if f.read(8) != MAGIC:
            raise ValueError(f"{path}: not a grid checkpoint")
        (hl,) = struct.unpack("<I", f.read(4))
        head = json.loads(f.read(hl).decode())
        payload = f.read()
    n, wpr = head["n"], head["words_per_row"]
    if wpr != words_per_row(n) or len(payload) != n * wpr * 8:
        raise ValueError(f"{path}: truncated or inconsistent checkpoint")
    if hashlib.sha256(payload).hexdigest() != head["payload_sha256"]:
        raise ValueError(f"{path}: checksum mismatch")
    return head, np.frombuffer(payload, dtype="<u8").reshape(n, wpr).copy()


def save(path, solver, generation=0, meta=None):
    """Write `solver`'s current grid.  Packs on the device (ltl_pack_device) and
    downloads the packed words only."""
    import torch
    from . import ltl
    n = solver.n
    wpr = words_per_row(n)
    dev = torch.device("cuda", solver.device)
    cells = torch.empty((n, n), dtype=torch.uint8, device=dev)
    words = torch.empty((n, wpr), dtype=torch.int64, device=dev)
    torch.cuda.synchronize(dev)
    solver.download_device(cells.data_ptr(), n)
    solver.synchronize()
    ltl.check(ltl.lib().ltl_pack_device(ctypes.c_void_p(cells.data_ptr()), n, n, n,
                                        ctypes.c_void_p(words.data_ptr()), wpr * 8, None))
    torch.cuda.synchronize(dev)
    host = words.cpu().numpy().view("<u8")
    write(path, host, n, solver.radius, solver.rule, generation, meta)


def load(path, solver=None, variant=None, device=0):
    """Restore a checkpoint into `solver` (same n), or into a new CUDASolver built
    from the header.  Returns (solver, header)."""
    import torch
    from . import ltl
    head, host = read(path)
    n = head["n"]
    if solver is None:
        kw = {} if variant is None else {"variant": variant}
        solver = ltl.CUDASolver(n, head["radius"], tuple(head["rule"]), device=device, **kw)
    elif solver.n != n:
        raise ValueError(f"checkpoint holds n={n}, solver has n={solver.n}")
    dev = torch.device("cuda", solver.device)
    words = torch.from_numpy(host.view(np.int64)).to(dev)
    cells = torch.empty((n, n), dtype=torch.uint8, device=dev)
    ltl.check(ltl.lib().ltl_unpack_device(ctypes.c_void_p(words.data_ptr()), head["words_per_row"] * 8, n, n,
                                          ctypes.c_void_p(cells.data_ptr()), n, None))
    torch.cuda.synchronize(dev)
    solver.upload_device(cells.data_ptr(), n)
    solver.synchronize()
    return solver, head
