"""Host-side mirror of the reference's FLOW application interface over libymflow.

Names follow the reference so code and tests read alike:

  GluonField        device-resident Field<SU3,4> (include/Math/field.h:52-76)
  SuperObs          plaq / energy / topc observable (include/Observables/superobs.h)
  WilsonFlow        the FLOW app (include/Apps/wilsonflow.h): applyWilsonFlow,
                    flowConfigurations, with the reference's step schedule
  read_conf         LatticeIO::InputConf::readConf (src/InputOutput/inputconf.cpp:114-155)
  get_input_list    InputConf::getInputList (inputconf.cpp:76-82)
  write_flow_obs    LatticeIO::OutputObs::writeFlowObs (src/InputOutput/outputobs.cpp:64-84)

Every computation runs in libymflow.so on the GPU; there is no CPU path.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path
from typing import Iterable, List, Sequence

import numpy as np

from . import _native as N


def _dims(size: Sequence[int]):
    if len(size) != 4:
        raise ValueError("lattice size must have 4 extents (x, y, z, t)")
    return N._I4(*[int(v) for v in size])


def volume(size: Sequence[int]) -> int:
    return int(size[0]) * int(size[1]) * int(size[2]) * int(size[3])


def read_conf(path, size: Sequence[int], big_endian: bool = False) -> np.ndarray:
    """Links of a .bin configuration: raw doubles, per global site (x fastest) 4
    links of 18 doubles (inputconf.cpp:114-155); big_endian reads the
    byte-reversed "Chroma" variant (inputconf.cpp:135-143).  Shape
    (Nt, Nz, Ny, Nx, 4, 18), native byte order."""
    n = volume(size) * 4 * 18
    a = np.fromfile(str(path), dtype=">f8" if big_endian else "<f8")
    if a.size != n:
        raise ValueError(f"{path}: {a.size * 8} bytes, expected {n * 8} for lattice {tuple(size)}")
    return a.astype(np.float64).reshape(size[3], size[2], size[1], size[0], 4, 18)


def write_conf(path, links: np.ndarray, big_endian: bool = False) -> None:
    """Writes links in the .bin layout read_conf reads (the reference's writer
    is a no-op, src/InputOutput/outputconf.cpp:102)."""
    np.ascontiguousarray(links, dtype=">f8" if big_endian else "<f8").tofile(str(path))


def get_input_list(input_dir) -> List[str]:
    """Every *.bin in input_dir, sorted by path (inputconf.cpp:76-82)."""
    return sorted(str(p) for p in Path(input_dir).iterdir() if p.suffix == ".bin")


def write_flow_obs(output_dir, conf_num: int, matrix: Iterable[Sequence[float]]) -> Path:
    """OutputDir/flow/confNNNN.dat with the header and "%lf\\t" rows of
    src/InputOutput/outputobs.cpp:64-84 (columns t, plaq, topc, energy)."""
    d = Path(output_dir) / "flow"
    d.mkdir(parents=True, exist_ok=True)
    p = d / ("conf%04d.dat" % conf_num)
    with open(p, "w") as f:
        f.write("Flow Time\tPlaq.\tTopc.\tEnerg.\t\n")
        for row in matrix:
            f.write("".join("%f\t" % v for v in row) + "\n")
    return p


class GluonField:
    """A gauge field resident on one B200, in one of the three storage forms
    ("fp64", "fp32_18", "fp32_12")."""

    def __init__(self, size: Sequence[int], precision: str = "fp64", device: int = 0):
        self.size = tuple(int(v) for v in size)
        self.precision = precision
        prec = N.PRECISIONS[precision]
        lib = N.load()
        st = ctypes.c_int(0)
        self._ctx = lib.ymflow_create(_dims(self.size), prec, int(device), ctypes.byref(st))
        if not self._ctx:
            raise N.YmflowError(st.value, lib.ymflow_last_error(None).decode(errors="replace"))
        self.sites = volume(self.size)

    @classmethod
    def slab(cls, global_size: Sequence[int], t0: int, nt: int, precision: str = "fp64",
             device: int = 0) -> "GluonField":
        """Time slices [t0, t0 + nt) of a configuration of extents global_size,
        with one halo slice on each side (the reference's domain decomposition,
        src/ParallelTools/parallel.cpp:57-100, along t).  upload/download and
        friends address the slab's own sites: the .bin file's sites
        [t0 Vs, (t0 + nt) Vs).  Flow it with connect() + flow() (one process
        per GPU) or with slab_group_flow() (all slabs in this process)."""
        self = cls.__new__(cls)
        g = tuple(int(v) for v in global_size)
        self.global_size = g
        self.t0, self.nt = int(t0), int(nt)
        self.size = (g[0], g[1], g[2], self.nt)
        self.precision = precision
        lib = N.load()
        st = ctypes.c_int(0)
        self._ctx = lib.ymflow_create_slab(_dims(g), self.t0, self.nt, N.PRECISIONS[precision], int(device),
                                           ctypes.byref(st))
        if not self._ctx:
            raise N.YmflowError(st.value, lib.ymflow_last_error(None).decode(errors="replace"))
        self.sites = volume(self.size)
        return self

    @classmethod
    def block(cls, global_size: Sequence[int], origin: Sequence[int], extent: Sequence[int],
              precision: str = "fp64", device: int = 0) -> "GluonField":
        """Sites [origin, origin + extent) of a configuration of extents
        global_size, with one halo layer on each side of every split direction
        (the reference's Cartesian domain decomposition,
        src/ParallelTools/parallel.cpp:57-100).  upload/download address the
        block's own sites in lexicographic order over `extent`.  Flow it with
        block_group_flow()."""
        self = cls.__new__(cls)
        g = tuple(int(v) for v in global_size)
        self.global_size = g
        self.origin = tuple(int(v) for v in origin)
        self.size = tuple(int(v) for v in extent)
        self.precision = precision
        lib = N.load()
        st = ctypes.c_int(0)
        self._ctx = lib.ymflow_create_block(_dims(g), _dims(self.origin), _dims(self.size),
                                            N.PRECISIONS[precision], int(device), ctypes.byref(st))
        if not self._ctx:
            raise N.YmflowError(st.value, lib.ymflow_last_error(None).decode(errors="replace"))
        self.sites = volume(self.size)
        return self

    def connect(self, nccl_id: bytes, rank: int, nranks: int, lower: int, upper: int) -> None:
        """Joins the NCCL communicator of nccl_id (from nccl_unique_id() on rank
        0); lower/upper are the ranks holding the neighbouring slices."""
        if len(nccl_id) != N.NCCL_ID_BYTES:
            raise ValueError("an NCCL id has 128 bytes")
        _prefer_framework_nccl()
        buf = ctypes.create_string_buffer(bytes(nccl_id), N.NCCL_ID_BYTES)
        self._check(N.load().ymflow_slab_connect(self.ctx, buf, int(rank), int(nranks), int(lower), int(upper)))

    # lifetime
    def close(self) -> None:
        if getattr(self, "_ctx", None):
            N.load().ymflow_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def ctx(self):
        if not self._ctx:
            raise RuntimeError("GluonField is closed")
        return self._ctx

    def _check(self, status: int) -> None:
        N.check(status, self.ctx)

    # data movement
    def upload(self, links: np.ndarray) -> None:
        a = np.ascontiguousarray(links, dtype=np.float64)
        if a.size != self.sites * 72:
            raise ValueError("links must hold 4*V*18 doubles")
        self._check(N.load().ymflow_upload(self.ctx, a.ctypes.data))

    def download(self) -> np.ndarray:
        a = np.empty((self.size[3], self.size[2], self.size[1], self.size[0], 4, 18), dtype=np.float64)
        self._check(N.load().ymflow_download(self.ctx, a.ctypes.data))
        return a

    def upload_sites(self, links: np.ndarray, first_site: int) -> None:
        """Sites [first_site, first_site + n) from a .bin-layout block of n*72
        doubles, little- or big-endian (">f8": byte-reversed on the device)."""
        a = np.ascontiguousarray(links)
        if a.dtype not in (np.dtype("<f8"), np.dtype(">f8")) or a.size % 72:
            raise ValueError("links must be float64 with 72 doubles per site")
        flags = N.IO_BIG_ENDIAN if a.dtype.byteorder == ">" else 0
        self._check(N.load().ymflow_upload_sites(self.ctx, a.ctypes.data, int(first_site), a.size // 72, flags))

    def download_sites(self, first_site: int, nsites: int, big_endian: bool = False) -> np.ndarray:
        a = np.empty((int(nsites), 4, 18), dtype=">f8" if big_endian else "<f8")
        flags = N.IO_BIG_ENDIAN if big_endian else 0
        self._check(N.load().ymflow_download_sites(self.ctx, a.ctypes.data, int(first_site), int(nsites), flags))
        return a

    def load_conf(self, path, big_endian: bool = False, chunk_sites: int = 65536) -> None:
        """Loads a .bin file (this context's part of it, for a slab) through the
        library's double-buffered reader: no whole-field host copy."""
        flags = N.IO_BIG_ENDIAN if big_endian else 0
        self._check(N.load().ymflow_load_file(self.ctx, str(path).encode(), flags, int(chunk_sites)))

    def init_links(self, kind: str = "expiah", a: float = 0.35, seed: int = 1, config: int = 0,
                   haar_frac: float = 0.0) -> None:
        k = {"cold": N.FIELD_COLD, "expiah": N.FIELD_EXPIAH}[kind]
        self._check(N.load().ymflow_init_links(self.ctx, k, float(a), int(seed), int(config), float(haar_frac)))

    def generate_metropolis(self, beta: float, su3eps: float = 0.24, sweeps: int = 200, hits: int = 30,
                            seed: int = 1, start: str = "cold") -> float:
        """Metropolis generation of the Wilson action (the reference's
        GaugeFieldFactory update, src/Apps/gaugefieldfactory.cpp:192-220);
        returns the acceptance."""
        k = {"cold": N.FIELD_COLD, "hot": N.FIELD_HOT, "current": N.FIELD_CURRENT}[start]
        acc = ctypes.c_double(0)
        self._check(N.load().ymflow_generate_metropolis(self.ctx, k, float(beta), float(su3eps), int(sweeps),
                                                        int(hits), int(seed), ctypes.byref(acc)))
        return acc.value

    # compute
    def observables(self) -> N.Obs:
        o = N.Obs()
        self._check(N.load().ymflow_observables(self.ctx, ctypes.byref(o)))
        return o

    def flow(self, eps: float, nsteps: int, measure_every: int = 1, reunit_every: int = 0) -> np.ndarray:
        """nsteps RK3 steps; rows (step, t, plaq, topc, energy, t2E)."""
        rows = 1 + sum(1 for s in range(1, nsteps + 1)
                       if (measure_every > 0 and s % measure_every == 0) or s == nsteps)
        out = (N.Obs * rows)()
        n = ctypes.c_int(0)
        self._check(N.load().ymflow_flow(self.ctx, float(eps), int(nsteps), int(measure_every), int(reunit_every),
                                         out, rows, ctypes.byref(n)))
        return np.array([out[i].as_tuple() for i in range(n.value)])

    def derivative(self, mu: int) -> np.ndarray:
        """Z_mu at every site, shape (V, 18): PureGauge::computeDerivative(mu)."""
        z = np.empty((self.sites, 18), dtype=np.float64)
        self._check(N.load().ymflow_derivative(self.ctx, int(mu), z.ctypes.data))
        return z

    def reset_time(self) -> None:
        self._check(N.load().ymflow_reset_time(self.ctx))

    def set_time(self, step: int, t: float) -> None:
        """Resume the step and flow-time counters (after re-uploading a checkpoint)."""
        self._check(N.load().ymflow_set_time(self.ctx, int(step), float(t)))

    def time_steps(self, eps: float, nsteps: int, kernels: bool = False):
        """(elapsed_ms, kernel_ms or None) of nsteps device-timed RK3 steps."""
        el = ctypes.c_float(0)
        km = ctypes.c_float(0)
        self._check(N.load().ymflow_time_steps(self.ctx, float(eps), int(nsteps), ctypes.byref(el),
                                               ctypes.byref(km) if kernels else None))
        return el.value, (km.value if kernels else None)

    def time_kernels(self, eps: float, nsteps: int):
        """(elapsed_ms, plaquette-field kernels ms, stage kernels ms) of nsteps
        device-timed RK3 steps, each kernel kind summed over its launches."""
        el, fm, sm = ctypes.c_float(0), ctypes.c_float(0), ctypes.c_float(0)
        self._check(N.load().ymflow_time_kernels(self.ctx, float(eps), int(nsteps), ctypes.byref(el),
                                                 ctypes.byref(fm), ctypes.byref(sm)))
        return el.value, fm.value, sm.value

    def set_option(self, key: int, value: int) -> None:
        self._check(N.load().ymflow_set_option(self.ctx, int(key), int(value)))

    def get_option(self, key: int) -> int:
        v = ctypes.c_int64(0)
        self._check(N.load().ymflow_get_option(self.ctx, int(key), ctypes.byref(v)))
        return v.value

    def autotune(self, eps: float = 0.01):
        """Times every stage form and tiling on this lattice and keeps the
        fastest (cached per extents and precision); returns (form, ty, tz)."""
        f, ty, tz = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
        self._check(N.load().ymflow_autotune(self.ctx, float(eps), ctypes.byref(f), ctypes.byref(ty),
                                             ctypes.byref(tz)))
        return f.value, ty.value, tz.value

    def set_tile(self, ty: int, tz: int, lpt: int = 4, lean: int = 0) -> None:
        """The shared-memory stage kernel's tile (form 2), and that form:
        ty x tz x-lines per tile, lpt links per thread, lean = the 64-register
        kernel."""
        self.set_option(N.OPT_TILE, tile_option(ty, tz, lpt, lean))
        self.set_option(N.OPT_STAGE_FORM, N.STAGE_TILE)

    def device_bytes(self) -> int:
        b = ctypes.c_int64(0)
        self._check(N.load().ymflow_device_bytes(self.ctx, ctypes.byref(b)))
        return b.value


class Ensemble:
    """Many configurations (any mix of lattice sizes) flowed together on one GPU:
    one persistent launch per RK3 stage for all of them, steps replayed as a
    CUDA graph.  The batched form of WilsonFlow::flowConfigurations
    (src/Apps/wilsonflow.cpp:96-109)."""

    def __init__(self, sizes: Sequence[Sequence[int]], precision: str = "fp32_18", device: int = 0):
        self.sizes = [tuple(int(v) for v in s) for s in sizes]
        dims = (ctypes.c_int * (4 * len(self.sizes)))(*[v for s in self.sizes for v in s])
        st = ctypes.c_int(0)
        lib = N.load()
        self._ens = lib.ymflow_ensemble_create(len(self.sizes), dims, N.PRECISIONS[precision], int(device),
                                               ctypes.byref(st))
        if not self._ens:
            raise N.YmflowError(st.value, lib.ymflow_ensemble_last_error(None).decode(errors="replace"))
        self.precision = precision

    def close(self) -> None:
        if getattr(self, "_ens", None):
            N.load().ymflow_ensemble_destroy(self._ens)
            self._ens = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, status: int) -> None:
        if status != N.OK:
            raise N.YmflowError(status, N.load().ymflow_ensemble_last_error(self._ens).decode(errors="replace"))

    def upload(self, conf: int, links: np.ndarray) -> None:
        a = np.ascontiguousarray(links, dtype=np.float64)
        if a.size != volume(self.sizes[conf]) * 72:
            raise ValueError("links must hold 4*V*18 doubles")
        self._check(N.load().ymflow_ensemble_upload(self._ens, int(conf), a.ctypes.data))

    def download(self, conf: int) -> np.ndarray:
        n = self.sizes[conf]
        a = np.empty((n[3], n[2], n[1], n[0], 4, 18), dtype=np.float64)
        self._check(N.load().ymflow_ensemble_download(self._ens, int(conf), a.ctypes.data))
        return a

    def init_links(self, conf: int, kind: str = "expiah", a: float = 0.35, seed: int = 1, config: int = 0,
                   haar_frac: float = 0.0) -> None:
        k = {"cold": N.FIELD_COLD, "expiah": N.FIELD_EXPIAH}[kind]
        self._check(N.load().ymflow_ensemble_init_links(self._ens, int(conf), k, float(a), int(seed), int(config),
                                                        float(haar_frac)))

    def flow(self, eps: float, nsteps: int, measure_every: int = 0, reunit_every: int = 0) -> np.ndarray:
        """rows x nconf x (step, t, plaq, topc, energy, t2E)."""
        rows = 1 + sum(1 for s in range(1, nsteps + 1)
                       if (measure_every > 0 and s % measure_every == 0) or s == nsteps)
        nc = len(self.sizes)
        out = (N.Obs * (rows * nc))()
        n = ctypes.c_int(0)
        self._check(N.load().ymflow_ensemble_flow(self._ens, float(eps), int(nsteps), int(measure_every),
                                                  int(reunit_every), out, rows, ctypes.byref(n)))
        return np.array([out[i].as_tuple() for i in range(n.value * nc)]).reshape(n.value, nc, 6)

    def time_steps(self, eps: float, nsteps: int) -> float:
        ms = ctypes.c_float(0)
        self._check(N.load().ymflow_ensemble_time_steps(self._ens, float(eps), int(nsteps), ctypes.byref(ms)))
        return ms.value

    def autotune(self, eps: float = 0.01):
        b, g = ctypes.c_int(0), ctypes.c_int(0)
        self._check(N.load().ymflow_ensemble_autotune(self._ens, float(eps), ctypes.byref(b), ctypes.byref(g)))
        return b.value, g.value

    def set_tuning(self, stage_form: int, block: int = 128, grid: int = 0) -> None:
        """Chooses the stage form by hand (see ymflow_ensemble_set_tuning)."""
        self._check(N.load().ymflow_ensemble_set_tuning(self._ens, int(stage_form), int(block), int(grid)))

    def tuning(self):
        """(stage form, block, grid) the ensemble flows with."""
        f, b, g = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
        self._check(N.load().ymflow_ensemble_tuning(self._ens, ctypes.byref(f), ctypes.byref(b), ctypes.byref(g)))
        return f.value, b.value, g.value

    def reset_time(self) -> None:
        self._check(N.load().ymflow_ensemble_reset_time(self._ens))


def tile_option(ty: int, tz: int, lpt: int = 4, lean: int = 0) -> int:
    """YMFLOW_OPT_TILE's value of a tiling."""
    return (int(lean) << 36) | (int(lpt) << 32) | (int(ty) << 16) | int(tz)


def _prefer_framework_nccl() -> None:
    """Point the library at the NCCL that PyTorch ships (without importing
    torch), so that torch imported later in this process finds the NCCL it was
    built against already loaded."""
    import importlib.util
    import os

    if os.environ.get("YMFLOW_NCCL_LIB"):
        return
    spec = importlib.util.find_spec("nvidia.nccl")
    for root in (spec.submodule_search_locations or []) if spec else []:
        lib = Path(root) / "lib" / "libnccl.so.2"
        if lib.exists():
            os.environ["YMFLOW_NCCL_LIB"] = str(lib)
            return


def nccl_unique_id() -> bytes:
    """A fresh NCCL communicator id (128 bytes) for GluonField.connect."""
    _prefer_framework_nccl()
    buf = ctypes.create_string_buffer(N.NCCL_ID_BYTES)
    N.check(N.load().ymflow_nccl_unique_id(buf))
    return buf.raw


def slab_partition(nt_global: int, nranks: int, rank: int):
    """(t0, nt, lower, upper) of rank's slab when nt_global time slices are
    split over nranks ranks as evenly as possible, ranks in time order."""
    if not 1 <= nranks <= nt_global or not 0 <= rank < nranks:
        raise ValueError("need 1 <= nranks <= time extent and 0 <= rank < nranks")
    base, extra = divmod(nt_global, nranks)
    t0 = rank * base + min(rank, extra)
    nt = base + (1 if rank < extra else 0)
    return t0, nt, (rank - 1) % nranks, (rank + 1) % nranks


def block_layout(global_size: Sequence[int], sub_size: Sequence[int]):
    """The reference's Cartesian decomposition of a lattice into sub-lattices
    of extents sub_size (src/ParallelTools/parallel.cpp:57-100): the grid
    (global / sub per direction) and each block's (origin, extent), block i at
    grid coordinates (i % grid[0], i / grid[0] % grid[1], ...), the order
    block_group_flow takes."""
    g = [int(v) for v in global_size]
    s = [int(v) for v in sub_size]
    if len(g) != 4 or len(s) != 4 or any(b < 1 or a % b for a, b in zip(g, s)):
        raise ValueError("every sub-lattice extent must divide the lattice extent")
    grid = [a // b for a, b in zip(g, s)]
    blocks = []
    for i in range(grid[0] * grid[1] * grid[2] * grid[3]):
        c, k = [], i
        for d in range(4):
            c.append(k % grid[d])
            k //= grid[d]
        blocks.append((tuple(c[d] * s[d] for d in range(4)), tuple(s)))
    return grid, blocks


def block_halo_plan(grid: Sequence[int], index: int, local_size: Sequence[int]):
    """The halo exchange of block `index` after every stage, as the library's
    block groups run it: one phase per split direction d (grid[d] > 1) in order
    x, y, z, t; in each, the block's first own layer (local coordinate 1)
    goes to the lower neighbour's upper halo and its last (local_size[d] - 2)
    to the upper neighbour's lower halo, whole faces including the halo layers
    of the directions exchanged before.  Each entry: direction, the neighbour
    block of each side, and the local coordinates sent and received."""
    stride = [1, grid[0], grid[0] * grid[1], grid[0] * grid[1] * grid[2]]
    plan = []
    for d in range(4):
        if grid[d] < 2:
            continue
        c = (index // stride[d]) % grid[d]
        lower = index + (((c - 1) % grid[d]) - c) * stride[d]
        upper = index + (((c + 1) % grid[d]) - c) * stride[d]
        n = int(local_size[d])
        plan.append({"dir": d, "lower": lower, "upper": upper,
                     "send_to_lower": 1, "send_to_upper": n - 2, "recv_from_lower": 0, "recv_from_upper": n - 1})
    return plan


def block_group_flow(blocks: Sequence[GluonField], grid: Sequence[int], eps: float, nsteps: int,
                     measure_every: int = 1, reunit_every: int = 0) -> np.ndarray:
    """ymflow_flow over the blocks of one configuration held in this process
    (in block_layout's order); rows (step, t, plaq, topc, energy, t2E) of the
    whole configuration."""
    rows = 1 + sum(1 for s in range(1, nsteps + 1)
                   if (measure_every > 0 and s % measure_every == 0) or s == nsteps)
    out = (N.Obs * rows)()
    n = ctypes.c_int(0)
    arr = (ctypes.c_void_p * len(blocks))(*[f.ctx for f in blocks])
    N.check(N.load().ymflow_block_group_flow(arr, len(blocks), _dims(grid), float(eps), int(nsteps),
                                             int(measure_every), int(reunit_every), out, rows, ctypes.byref(n)),
            blocks[0].ctx)
    return np.array([out[i].as_tuple() for i in range(n.value)])


def slab_halo_plan(nt: int):
    """The halo exchange of a time slab after every RK3 stage, in the posting
    order of the library's NCCL exchange (csrc/slab.cu): local slices are
    0 (lower halo), 1..nt (interior), nt + 1 (upper halo).  Each entry: the
    interior slice this rank sends and the neighbour it goes to, and the halo
    slice it receives and the neighbour that sends it.  A send of one entry
    lands in the receive of the same entry on the other side; `tag` numbers
    the entries, so that a rank that is the neighbour on both sides (two
    ranks) or its own neighbour (one) tells the two transfers apart.  It replaces shift()'s face exchange (include/Math/lattice.h:437-449)."""
    if nt < 1:
        raise ValueError("a slab holds at least one time slice")
    return [
        {"send_slice": 1, "to": "lower", "recv_slice": nt + 1, "from": "upper", "tag": 0},
        {"send_slice": nt, "to": "upper", "recv_slice": 0, "from": "lower", "tag": 1},
    ]


def slab_group_flow(slabs: Sequence[GluonField], eps: float, nsteps: int, measure_every: int = 1,
                    reunit_every: int = 0) -> np.ndarray:
    """ymflow_flow over the slabs of one configuration held in this process
    (in time order); rows (step, t, plaq, topc, energy, t2E) of the whole
    configuration."""
    rows = 1 + sum(1 for s in range(1, nsteps + 1)
                   if (measure_every > 0 and s % measure_every == 0) or s == nsteps)
    out = (N.Obs * rows)()
    n = ctypes.c_int(0)
    arr = (ctypes.c_void_p * len(slabs))(*[f.ctx for f in slabs])
    N.check(N.load().ymflow_slab_group_flow(arr, len(slabs), float(eps), int(nsteps), int(measure_every),
                                            int(reunit_every), out, rows, ctypes.byref(n)), slabs[0].ctx)
    return np.array([out[i].as_tuple() for i in range(n.value)])


def su3_exp(q: np.ndarray, device: int = 0) -> np.ndarray:
    """e^{iQ} of Hermitian traceless matrices (..., 18) on the GPU: exp(const SU3&)."""
    a = np.ascontiguousarray(q, dtype=np.float64).reshape(-1, 18)
    r = np.empty_like(a)
    st = N.load().ymflow_su3_exp(a.ctypes.data, r.ctypes.data, a.shape[0], int(device))
    if st != N.OK:
        raise N.YmflowError(st, "ymflow_su3_exp failed")
    return r


class SuperObs:
    """plaq, energy and topc of a field, as the reference's SuperObs
    (src/Observables/superobs.cpp:31-128)."""

    def __init__(self):
        self.plaq = self.energy = self.topc = float("nan")
        self._field = None

    def initObservable(self, field: GluonField) -> None:
        self._field = field

    def compute(self) -> None:
        o = self._field.observables()
        self.plaq, self.energy, self.topc = o.plaq, o.energy, o.topc


class WilsonFlow:
    """The FLOW app (src/Apps/wilsonflow.cpp) over libymflow."""

    def __init__(self, tauFinal: float, epsilon: float):
        self.m_tauFinal = float(tauFinal)
        self.m_epsilon = float(epsilon)
        self.field: GluonField | None = None

    def createLattice(self, size: Sequence[int], precision: str = "fp64", device: int = 0) -> None:
        self.field = GluonField(size, precision, device)

    def nrows(self) -> int:
        """int(tauFinal/epsilon) rows: row 0 at t = 0, then one per flow step,
        hence int(tauFinal/epsilon) - 1 steps (src/Apps/wilsonflow.cpp:117,124)."""
        return int(self.m_tauFinal / self.m_epsilon)

    def applyWilsonFlow(self) -> np.ndarray:
        """Flows the loaded field; rows (t, plaq, topc, energy) as flowObsMatrix
        (src/Apps/wilsonflow.cpp:115-136)."""
        nsteps = max(self.nrows() - 1, 0)
        self.field.reset_time()
        rows = self.field.flow(self.m_epsilon, nsteps, measure_every=1)
        return rows[: max(self.nrows(), 1), [1, 2, 3, 4]]

    def flowConfigurations(self, input_dir, output_dir) -> List[Path]:
        """Every sorted *.bin of input_dir: read, flow, write flow/confNNNN.dat
        (src/Apps/wilsonflow.cpp:96-109)."""
        written = []
        for conf_num, path in enumerate(get_input_list(input_dir)):
            self.field.upload(read_conf(path, self.field.size))
            written.append(write_flow_obs(output_dir, conf_num, self.applyWilsonFlow()))
        return written
