"""One grid split into row strips, one strip per GPU (or several in one process).

The reference steps one grid in one process; this splits an n x n torus by
rows.  Strip p owns inner rows [a_p, b_p) (m_p rows) and is held as a torus of
its own with m_p + 2h rows, h = R * k: h halo rows above and below.  Each
generation the rows a strip cannot know (its halo edges, where its own torus
wraps falsely) spoil R more rows from each end, so after k generations exactly
the h halo rows are stale and the m inner rows are exact.  h/m of the step work
is redone in the halos.

Every block of k generations (ring neighbours on the torus):

  1. the strip's new boundary rows -- its first and last h inner rows after
     the block, which the neighbours need as halos for the next block -- come
     first, from two small edge tori of 3h rows each (copies of its top and
     bottom 3h rows, stepped k generations: their middle h rows are exact);
  2. they go out (first rows to the strip above, last rows to the strip
     below), and the neighbours' boundary rows are received as the new halos;
  3. meanwhile the strip itself steps the k generations;
  4. the received rows replace its (now stale) halo rows.

With NCCL the transfer of step 2 runs on NCCL's own stream while the kernels
of step 3 run on the strip's: the exchange is hidden behind the block's
compute, at the price of stepping 2 x 3h extra rows.  Each exchange moves 2h
rows of n bytes per strip.

Two transports:
  LocalStrips  all strips in one process (tests, or several strips on one
               device), exchanged by tensor copies;
  DistStrips   one strip per torch.distributed rank (NCCL between GPUs, gloo on
               CPU), exchanged with batched isend/irecv between ring neighbours.

A strip is stepped by a "stepper": an object with `rows`, `n`, `read_rows(row0,
nrows, out)`, `write_rows(row0, src)` (torch tensors of shape (nrows, n)) and
`step(g)`.  GpuStepper wraps a rectangular plain or bit-packed context
(ltl_create_rect_variant, ltl_download_rows_device / ltl_upload_rows_device).
"""
import torch


def partition(n, parts):
    """Row bounds [(a, b)] of `parts` balanced strips of an n-row grid."""
    return [(p * n // parts, (p + 1) * n // parts) for p in range(parts)]


def halo_rows(radius, k):
    return radius * k


class GpuStepper:
    """A strip as a rows x n torus on one GPU (plain or bit-packed variant),
    ordered on the current torch stream, which must not be the legacy default
    stream: its handle (0) would select the context's own stream, unordered with
    torch's work.  The drivers below build their steppers inside a stream of
    their own."""

    def __init__(self, rows, n, radius, rule, device=0, variant=None):
        from .ltl import CUDASolver, VARIANT_PLAIN
        stream = torch.cuda.current_stream(device)
        if stream.cuda_stream == 0:
            raise RuntimeError("GpuStepper needs a non-default current stream (use torch.cuda.stream(...))")
        self.rows, self.n = rows, n
        self.solver = CUDASolver(n, radius, rule, variant=VARIANT_PLAIN if variant is None else variant,
                                 device=device, rows=rows)
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
    def __init__(self, a, b, h, stepper, top=None, bottom=None):
        self.a, self.b, self.h, self.st = a, b, h, stepper
        self.m = b - a
        self.top, self.bottom = top, bottom  # edge tori of 3h rows (overlapped exchange)


class _Base:
    """Shared logic: loading the global grid, the block schedule, gathering.
    On a CUDA device all work (the steppers', the copies, the exchanges) is
    ordered on one stream of the driver's own, `self.stream`.  overlap=False
    steps the strip first and reads its boundary rows from it afterwards (no
    edge tori, nothing to hide the exchange behind)."""

    def __init__(self, n, radius, k, device, overlap=True):
        if k < 1:
            raise ValueError("k (generations per exchange) must be >= 1")
        self.n, self.radius, self.k = n, radius, k
        self.h = halo_rows(radius, k)
        self.overlap = overlap
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

    def _strip(self, a, b, make_stepper):
        h, n = self.h, self.n
        st = make_stepper(b - a + 2 * h, n)
        if not self.overlap:
            return _Strip(a, b, h, st)
        return _Strip(a, b, h, st, make_stepper(3 * h, n), make_stepper(3 * h, n))

    def _rows(self, count):
        return torch.empty((count, self.n), dtype=torch.uint8, device=self.device)

    def _load(self, s, grid):
        """Strip s's local rows (inner rows a-h .. b+h, modulo n) from a global grid tensor."""
        idx = torch.arange(s.a - s.h, s.b + s.h, device=grid.device) % self.n
        s.st.write_rows(0, grid.index_select(0, idx).contiguous())

    def _boundary_ahead(self, s, g):
        """Strip s's first and last h inner rows as they will be after g <= k
        generations, from its edge tori (local rows [0, 3h) and [m - h, m + 2h))."""
        h = self.h
        buf, first, last = self._rows(3 * h), self._rows(h), self._rows(h)
        s.st.read_rows(0, 3 * h, buf)
        s.top.write_rows(0, buf)
        s.top.step(g)
        s.top.read_rows(h, h, first)
        s.st.read_rows(s.m - h, 3 * h, buf)
        s.bottom.write_rows(0, buf)
        s.bottom.step(g)
        s.bottom.read_rows(h, h, last)
        return first, last

    def _boundary_now(self, s):
        """Strip s's first and last h inner rows, read from the strip itself."""
        first, last = self._rows(self.h), self._rows(self.h)
        s.st.read_rows(self.h, self.h, first)
        s.st.read_rows(s.m, self.h, last)
        return first, last

    def step(self, generations):
        with self._on_stream():
            left = generations
            while left > 0:
                g = min(self.k, left)
                self._block(g)
                left -= g

    def close(self):
        """Release every stepper that has a close() (the GPU contexts)."""
        for s in self._local():
            for st in (s.st, s.top, s.bottom):
                if st is not None and hasattr(st, "close"):
                    st.close()


class LocalStrips(_Base):
    """All strips in this process: `make_stepper(rows, n)` builds each strip's stepper."""

    def __init__(self, n, radius, parts, k, make_stepper, device="cpu", overlap=True):
        super().__init__(n, radius, k, device, overlap)
        bounds = partition(n, parts)
        self._check(bounds)
        with self._on_stream():
            self.strips = [self._strip(a, b, make_stepper) for a, b in bounds]

    def _local(self):
        return self.strips

    def set_state(self, grid):
        with self._on_stream():
            g = torch.as_tensor(grid, dtype=torch.uint8).to(self.device)
            for s in self.strips:
                self._load(s, g)

    def _block(self, g):
        P, h = len(self.strips), self.h
        if self.overlap:
            bounds = [self._boundary_ahead(s, g) for s in self.strips]
            for s in self.strips:
                s.st.step(g)
        else:
            for s in self.strips:
                s.st.step(g)
            bounds = [self._boundary_now(s) for s in self.strips]
        for p, s in enumerate(self.strips):
            s.st.write_rows(0, bounds[(p - 1) % P][1])      # above me: the previous strip's last rows
            s.st.write_rows(s.m + h, bounds[(p + 1) % P][0])  # below me: the next strip's first rows

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

    def __init__(self, n, radius, k, make_stepper, device, group=None, overlap=True):
        import torch.distributed as dist
        super().__init__(n, radius, k, device, overlap)
        self.dist, self.group = dist, group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        bounds = partition(n, self.world)
        self._check(bounds)
        self.bounds = bounds
        a, b = bounds[self.rank]
        with self._on_stream():
            self.s = self._strip(a, b, make_stepper)

    def _local(self):
        return [self.s]

    def set_state(self, grid):
        """Every rank passes the same global grid (or at least the rows of its strip and halos)."""
        with self._on_stream():
            self._load(self.s, torch.as_tensor(grid, dtype=torch.uint8).to(self.device))

    def _post(self, first, last):
        """Send my first rows up and my last rows down; receive the halo rows.
        Returns (requests, rows from the strip above, rows from the strip below)."""
        if self.world == 1:
            return [], last, first  # the torus wraps onto this strip itself
        up = (self.rank - 1) % self.world
        down = (self.rank + 1) % self.world
        from_up, from_down = self._rows(self.h), self._rows(self.h)
        d = self.dist
        # Per peer the messages match in issue order: my first rows go up, my last
        # rows go down; I receive the strip below's first rows, then the strip
        # above's last rows.  With two ranks both neighbours are the same peer and
        # that order pairs each message with the right halo.
        ops = [d.P2POp(d.isend, first, up, self.group), d.P2POp(d.isend, last, down, self.group),
               d.P2POp(d.irecv, from_down, down, self.group), d.P2POp(d.irecv, from_up, up, self.group)]
        return d.batch_isend_irecv(ops), from_up, from_down

    def _block(self, g):
        s = self.s
        if self.overlap:
            # the exchange is posted before the strip's own k generations are
            # enqueued, so that it runs beside them
            reqs, from_up, from_down = self._post(*self._boundary_ahead(s, g))
            s.st.step(g)
        else:
            s.st.step(g)
            reqs, from_up, from_down = self._post(*self._boundary_now(s))
        for req in reqs:
            req.wait()
        s.st.write_rows(0, from_up)
        s.st.write_rows(s.m + s.h, from_down)

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
