"""One grid split into row strips, one strip per GPU (or several in one process).

The reference steps one grid in one process; this splits an n x n torus by
rows.  Strip p owns inner rows [a_p, b_p) (m_p rows) and is held as a torus of
its own with m_p + 2h rows, h = R * k: h halo rows above and below.  Every k
generations the strips exchange halos (ring neighbours on the torus):

    my inner rows [h, 2h)       -> the strip above, into its bottom halo
    my inner rows [m, m + h)    -> the strip below, into its top halo

and then step k generations on their own.  Each generation the rows a strip
cannot know (its halo edges, where its own torus wraps falsely) spoil R more
rows from each end, so after k generations exactly the h halo rows are stale
and the m inner rows are exact.  Each exchange moves 2h rows of n bytes per
strip; h/m of the step work is redone in the halos.

Two transports:
  LocalStrips  all strips in one process (tests, or several strips on one
               device), exchanged by tensor copies;
  DistStrips   one strip per torch.distributed rank (NCCL between GPUs, gloo on
               CPU), exchanged with batched isend/irecv between ring neighbours.

A strip is stepped by a "stepper": an object with `rows`, `n`, `read_rows(row0,
nrows, out)`, `write_rows(row0, src)` (torch tensors of shape (nrows, n)) and
`step(g)`.  GpuStepper wraps a rectangular plain-variant context
(ltl_create_rect, ltl_download_rows_device / ltl_upload_rows_device).
"""
import torch


def partition(n, parts):
    """Row bounds [(a, b)] of `parts` balanced strips of an n-row grid."""
    return [(p * n // parts, (p + 1) * n // parts) for p in range(parts)]


def halo_rows(radius, k):
    return radius * k


class GpuStepper:
    """A strip as a rows x n torus on one GPU (plain variant), ordered on the
    current torch stream, which must not be the legacy default stream: its
    handle (0) would select the context's own stream, unordered with torch's
    work.  The drivers below build their steppers inside a stream of their own."""

    def __init__(self, rows, n, radius, rule, device=0):
        from .ltl import CUDASolver
        stream = torch.cuda.current_stream(device)
        if stream.cuda_stream == 0:
            raise RuntimeError("GpuStepper needs a non-default current stream (use torch.cuda.stream(...))")
        self.rows, self.n = rows, n
        self.solver = CUDASolver(n, radius, rule, device=device, rows=rows)
        self.solver.set_stream(stream.cuda_stream)

    def read_rows(self, row0, nrows, out):
        self.solver.download_rows_device(row0, nrows, out.data_ptr(), self.n)

    def write_rows(self, row0, src):
        self.solver.upload_rows_device(row0, src.shape[0], src.data_ptr(), self.n)

    def step(self, g):
        self.solver.doSteps(g)

    def close(self):
        self.solver.close()


class _Strip:
    def __init__(self, a, b, h, stepper):
        self.a, self.b, self.h, self.st = a, b, h, stepper
        self.m = b - a


class _Base:
    """Shared logic: loading the global grid, stepping with exchanges, gathering.
    On a CUDA device all work (the steppers', the copies, the exchanges) runs on
    one stream of the driver's own, `self.stream`."""

    def __init__(self, n, radius, k, device):
        if k < 1:
            raise ValueError("k (generations per exchange) must be >= 1")
        self.n, self.radius, self.k = n, radius, k
        self.h = halo_rows(radius, k)
        self.device = torch.device(device)
        self.stream = torch.cuda.Stream(self.device) if self.device.type == "cuda" else None

    def _on_stream(self):
        import contextlib
        return torch.cuda.stream(self.stream) if self.stream is not None else contextlib.nullcontext()

    def _check(self, bounds):
        for a, b in bounds:
            if b - a < self.h:
                raise ValueError(f"strip of {b - a} rows is thinner than its halo ({self.h} = R * k rows): "
                                 f"use fewer strips or a smaller k")

    def _load(self, s, grid):
        """Strip s's local rows (inner rows a-h .. b+h, modulo n) from a global grid tensor."""
        idx = torch.arange(s.a - s.h, s.b + s.h, device=grid.device) % self.n
        s.st.write_rows(0, grid.index_select(0, idx).contiguous())

    def step(self, generations):
        with self._on_stream():
            left = generations
            while left > 0:
                g = min(self.k, left)
                self._exchange()
                for s in self._local():
                    s.st.step(g)
                left -= g


class LocalStrips(_Base):
    """All strips in this process: `make_stepper(rows, n)` builds each strip's stepper."""

    def __init__(self, n, radius, parts, k, make_stepper, device="cpu"):
        super().__init__(n, radius, k, device)
        bounds = partition(n, parts)
        self._check(bounds)
        with self._on_stream():
            self.strips = [_Strip(a, b, self.h, make_stepper(b - a + 2 * self.h, n)) for a, b in bounds]

    def _local(self):
        return self.strips

    def set_state(self, grid):
        with self._on_stream():
            g = torch.as_tensor(grid, dtype=torch.uint8).to(self.device)
            for s in self.strips:
                self._load(s, g)

    def _exchange(self):
        P, h, n = len(self.strips), self.h, self.n
        tops, bots = [], []
        for s in self.strips:
            t = torch.empty((h, n), dtype=torch.uint8, device=self.device)
            b = torch.empty((h, n), dtype=torch.uint8, device=self.device)
            s.st.read_rows(h, h, t)        # my first inner rows
            s.st.read_rows(s.m, h, b)      # my last inner rows
            tops.append(t)
            bots.append(b)
        for p, s in enumerate(self.strips):
            s.st.write_rows(0, bots[(p - 1) % P])          # above me: the previous strip's last rows
            s.st.write_rows(s.m + h, tops[(p + 1) % P])    # below me: the next strip's first rows

    def get_state(self):
        with self._on_stream():
            out = torch.empty((self.n, self.n), dtype=torch.uint8, device=self.device)
            for s in self.strips:
                s.st.read_rows(self.h, s.m, out[s.a:s.b])
        if self.stream is not None:
            torch.cuda.current_stream(self.device).wait_stream(self.stream)
        return out


class DistStrips(_Base):
    """One strip per rank of the default (or given) torch.distributed group.
    Tensors live on `device` (a CUDA device for NCCL, "cpu" for gloo)."""

    def __init__(self, n, radius, k, make_stepper, device, group=None):
        import torch.distributed as dist
        super().__init__(n, radius, k, device)
        self.dist, self.group = dist, group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        bounds = partition(n, self.world)
        self._check(bounds)
        self.bounds = bounds
        a, b = bounds[self.rank]
        with self._on_stream():
            self.s = _Strip(a, b, self.h, make_stepper(b - a + 2 * self.h, n))

    def _local(self):
        return [self.s]

    def set_state(self, grid):
        """Every rank passes the same global grid (or at least the rows of its strip and halos)."""
        with self._on_stream():
            self._load(self.s, torch.as_tensor(grid, dtype=torch.uint8).to(self.device))

    def _exchange(self):
        s, h, n = self.s, self.h, self.n
        up = (self.rank - 1) % self.world
        down = (self.rank + 1) % self.world
        top = torch.empty((h, n), dtype=torch.uint8, device=self.device)
        bot = torch.empty((h, n), dtype=torch.uint8, device=self.device)
        s.st.read_rows(h, h, top)
        s.st.read_rows(s.m, h, bot)
        if self.world == 1:
            s.st.write_rows(0, bot)
            s.st.write_rows(s.m + h, top)
            return
        from_up = torch.empty((h, n), dtype=torch.uint8, device=self.device)
        from_down = torch.empty((h, n), dtype=torch.uint8, device=self.device)
        d = self.dist
        # Per peer the messages match in issue order: my first rows go up, my last
        # rows go down; I receive the strip below's first rows, then the strip
        # above's last rows.  With two ranks both neighbours are the same peer and
        # that order pairs each message with the right halo.
        ops = [d.P2POp(d.isend, top, up, self.group), d.P2POp(d.isend, bot, down, self.group),
               d.P2POp(d.irecv, from_down, down, self.group), d.P2POp(d.irecv, from_up, up, self.group)]
        for req in d.batch_isend_irecv(ops):
            req.wait()
        s.st.write_rows(0, from_up)
        s.st.write_rows(s.m + h, from_down)

    def get_state(self):
        """The full grid on every rank (all-gather of the inner rows)."""
        with self._on_stream():
            out = self._gather()
        if self.stream is not None:
            torch.cuda.current_stream(self.device).wait_stream(self.stream)
        return out

    def _gather(self):
        s = self.s
        mine = torch.empty((s.m, self.n), dtype=torch.uint8, device=self.device)
        s.st.read_rows(self.h, s.m, mine)
        parts = [torch.empty((b - a, self.n), dtype=torch.uint8, device=self.device) for a, b in self.bounds]
        if self.world == 1:
            return mine
        # strips may differ in height by one row: gather padded to the largest
        mx = max(b - a for a, b in self.bounds)
        pad = torch.zeros((mx, self.n), dtype=torch.uint8, device=self.device)
        pad[:s.m] = mine
        got = [torch.empty_like(pad) for _ in range(self.world)]
        self.dist.all_gather(got, pad, group=self.group)
        for p, (a, b) in enumerate(self.bounds):
            parts[p] = got[p][:b - a]
        return torch.cat(parts, 0)
