"""Device pipeline of the line-by-line engine (host orchestration of the CUDA kernels).

One call of :func:`optical_depth` runs, on the current CUDA stream:

1. ``lbl_build_layers``  levels -> layers (or an upload of host layers)
2. ``lbl_layer_groups``  per (layer, line group) pressures, column, Q(296)/Q(T)
3. ``lbl_sort_lines``    reference band mask + sort by centre
4. ``lbl_gather_lines``  sorted line records
5. ``lbl_tile_ranges``   candidate lines of every reference tile
6. ``lbl_line_prep_*``   per (layer, line) strengths and widths
7. ``lbl_tau_tiles_*``   Voigt sums x R(nu, T) -> od[layer, nu]
8. ``lbl_layer_sum_exp_*`` (optional) column tau and exp(-tau/mu)

Host work is limited to what the reference does once per call in Python: the
(mol, iso) group selection with its warnings and errors
(``pylblrtm/forward.py:189-245``) and the grid and tile sizes
(``forward.py:141-142, 175-176``). Everything per line or per grid point runs on
the GPU. There is no CPU path.
"""

from __future__ import annotations

import ctypes
import math
import threading
import warnings
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _lib
from .atmosphere import COLUMN_FACTOR, P_STD_HPA
from .hitran_ids import MOL_ID_TO_NAME
from .spectral_data import SpectralData

INT_MAX = 2**31 - 1
# "fp32": multi-level float32 summation (default); "fp32-direct": float32 summation of
# every line at every point; "fp64": the plain float64 method.
PRECISIONS = ("fp32", "fp32-direct", "fp64")


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise _lib.EngineUnavailable(
            "no CUDA device is available; the line-by-line engine runs only on the GPU")
    return torch


@dataclass
class Group:
    """One (mol_id, iso_id) group that contributes, in reference order."""
    mol_id: int
    iso_id: int
    gas: str
    molar_mass: float
    tips_t: np.ndarray
    tips_q: np.ndarray


@dataclass
class Grid:
    """Uniform grid nu_i = nu_min + i*step and the reference tile size."""
    nu_min: float
    step: float
    n_nu: int
    tile_samples: int

    @property
    def nu(self) -> np.ndarray:
        nu = np.arange(self.n_nu, dtype=np.float64)      # nu_min + i * step, in place
        nu *= self.step
        nu += self.nu_min
        return nu

    def nu_at(self, i: int) -> float:
        return float(self.nu_min + np.float64(i) * self.step)


def make_grid(nu_min: float, nu_max: float, step: float, tile_width: float) -> Grid:
    """Grid size (forward.py:141) and tile size (forward.py:175-176)."""
    n = int(np.ceil((nu_max - nu_min) / step)) + 1
    return Grid(float(nu_min), float(step), n, tile_samples_for(float(nu_min), float(step), n, tile_width))


def tile_samples_for(nu_min: float, step: float, n_nu: int, tile_width: float) -> int:
    """Reference tile length: floor(tile_width / (nu[1]-nu[0]) + 1e-8), at least 1."""
    if n_nu > 1:
        nu01 = nu_min + np.arange(2, dtype=np.float64) * step
        eff = float(nu01[1] - nu01[0])
    else:
        eff = 0.001
    return max(1, int(np.floor(tile_width / eff + 1e-8)))


def grid_from_array(nu: np.ndarray, tile_width: float) -> Grid:
    """Recover (nu_min, step) from a grid array built as nu_min + arange(n)*step."""
    nu = np.asarray(nu, dtype=np.float64)
    if nu.ndim != 1 or nu.size < 1:
        raise ValueError("nu must be a non-empty 1-D array")
    n = nu.size
    if n == 1:
        return Grid(float(nu[0]), 0.001, 1, tile_samples_for(float(nu[0]), 0.001, 1, tile_width))
    d = float(nu[1] - nu[0])
    idx = np.arange(n, dtype=np.float64)
    for digits in (None, 15, 14, 13, 12, 11, 10, 9):
        s = d if digits is None else float(np.round(d, digits))
        if s > 0 and np.array_equal(nu[0] + idx * s, nu):
            return Grid(float(nu[0]), s, n, tile_samples_for(float(nu[0]), s, n, tile_width))
    raise ValueError("the GPU engine needs a uniform grid nu_min + arange(n) * step")


def select_groups(sd: SpectralData, profile_gases: Sequence[str], nu_first: float, nu_last: float,
                  cutoff: float, p_max: float, warn_level: int,
                  stats: Optional[dict] = None) -> Tuple[List[Group], np.ndarray]:
    """Host replica of the group selection of forward.py:189-245.

    Returns the contributing groups in sorted (mol_id, iso_id) order and the
    group index of every line (-1 for lines of skipped groups). Emits the same
    RuntimeWarnings and raises the same KeyError as the reference. ``stats``
    (a dict) receives "max_abs_shift", the largest finite |shift| (0 if none), and
    "band_lines", how many lines of the contributing groups pass the band mask (the
    host's count of the device sort's kept lines: the same comparisons, so never fewer).
    """
    lines = sd.lines
    mol = np.asarray(lines["mol_id"])
    iso = np.asarray(lines["iso_id"])
    n = np.asarray(lines["nu0"]).size
    gid = np.full(n, -1, dtype=np.int32)
    if stats is not None:
        stats["max_abs_shift"] = 0.0
        stats["band_lines"] = 0
    if n == 0:
        return [], gid
    # one native pass: distinct (mol, iso) pairs, band-mask counts (forward.py:190-191)
    # and each line's pair; ids must fit int32 (HITRAN numbers are small)
    for a in (mol, iso):
        if a.dtype != np.int32 and (a.min() < -2 ** 31 or a.max() >= 2 ** 31):
            raise ValueError("mol_id / iso_id values must fit a 32-bit integer")
    c = lambda a, t: np.ascontiguousarray(a, dtype=t)
    mol32, iso32 = c(mol, np.int32), c(iso, np.int32)
    nu0, shift = c(lines["nu0"], np.float64), c(lines["shift"], np.float64)
    pair_index = np.empty(n, dtype=np.int32)
    host = _lib.load_host()
    max_pairs = 256
    while True:
        pm = np.empty(max_pairs, np.int32)
        pi_ = np.empty(max_pairs, np.int32)
        pb = np.empty(max_pairs, np.int64)
        n_pairs = ctypes.c_int(0)
        smax = ctypes.c_double(-1.0)
        rc = host.lbl_line_pairs(mol32.ctypes.data, iso32.ctypes.data, nu0.ctypes.data, shift.ctypes.data, n,
                                 nu_first - cutoff, nu_last + cutoff, float(p_max), max_pairs, pm.ctypes.data,
                                 pi_.ctypes.data, pb.ctypes.data, ctypes.byref(n_pairs), pair_index.ctypes.data,
                                 ctypes.byref(smax))
        if rc == 0:
            break
        if max_pairs >= n:
            raise RuntimeError("lbl_line_pairs failed")
        max_pairs = min(n, 16 * max_pairs)
    k = n_pairs.value
    if stats is not None:
        stats["max_abs_shift"] = max(smax.value, 0.0)
    order = np.lexsort((pi_[:k], pm[:k]))                               # sorted (mol_id, iso_id)
    pairs = [(int(pm[j]), int(pi_[j])) for j in order]
    band_counts = pb[:k][order]
    groups: List[Group] = []
    lut_pairs: Dict[int, int] = {}
    for pi, (m, i) in enumerate(pairs):
        gas = MOL_ID_TO_NAME.get(int(m))
        if gas is None:
            warnings.warn(f"mol_id={m} is not in the HITRAN catalogue; lines skipped.",
                          RuntimeWarning, stacklevel=warn_level)
            continue
        if gas not in profile_gases:
            warnings.warn(
                f"Gas '{gas}' (mol_id={m}, iso_id={i}) is in the "
                f"spectral data but not in the atmospheric profile vmr; "
                f"its lines are skipped.", RuntimeWarning, stacklevel=warn_level)
            continue
        cnt = band_counts[pi]
        if cnt == 0:
            continue
        mm = sd.molar_masses.get((int(m), int(i)))
        if mm is None:
            warnings.warn(f"No molar mass found for (mol_id={m}, iso_id={i}); "
                          f"using dry-air mass as fallback.", RuntimeWarning, stacklevel=warn_level)
            mm = 28.97
        tkey = (int(m), int(i))
        if tkey not in sd.tips:
            raise KeyError(f"No TIPS data for (mol_id={m}, iso_id={i}). "
                           f"Available: {sorted(sd.tips.keys())}")
        t_arr, q_arr = sd.tips[tkey]
        if np.asarray(t_arr).size == 0 or np.asarray(t_arr).size != np.asarray(q_arr).size:
            raise ValueError("array of sample points is empty" if np.asarray(t_arr).size == 0
                             else "fp and xp are not of the same length.")
        lut_pairs[int(order[pi])] = len(groups)
        if stats is not None:
            stats["band_lines"] += int(cnt)
        groups.append(Group(int(m), int(i), gas, float(mm), np.asarray(t_arr, np.float64),
                            np.asarray(q_arr, np.float64)))
    if groups:
        lut = np.full(k, -1, dtype=np.int32)
        for j, g in lut_pairs.items():
            lut[j] = g
        if host.lbl_map_index(pair_index.ctypes.data, n, lut.ctypes.data, k, gid.ctypes.data) != 0:
            raise RuntimeError("lbl_map_index: pair index out of range")
    return groups, gid


def band_edges(nu_first: float, nu_last: float, cutoff: float,
               line_window: Optional[Tuple[float, float]] = None) -> Tuple[float, float]:
    """Edges of the device sort's band mask: the reference's nu[0] - cutoff and
    nu[-1] + cutoff (``forward.py:190-191, 215-220``), narrowed to a shard's line
    window when one is given."""
    lo, hi = nu_first - cutoff, nu_last + cutoff
    if line_window is not None:
        lo, hi = max(lo, float(line_window[0])), min(hi, float(line_window[1]))
    return lo, hi


@dataclass
class LayerInput:
    """Either levels (built into layers on the device) or ready layers."""
    gases: List[str]
    levels_p: Optional[np.ndarray] = None   # [n_prof, n_lev] hPa
    levels_t: Optional[np.ndarray] = None   # [n_prof, n_lev] K
    levels_vmr: Optional[np.ndarray] = None  # [n_prof, n_gas, n_lev]
    layer_p: Optional[np.ndarray] = None    # [n_prof, n_lay] atm
    layer_t: Optional[np.ndarray] = None
    layer_vmr: Optional[np.ndarray] = None  # [n_prof, n_gas, n_lay]
    layer_col: Optional[np.ndarray] = None

    @property
    def n_prof(self) -> int:
        return (self.levels_p if self.levels_p is not None else self.layer_p).shape[0]

    @property
    def n_lay(self) -> int:
        if self.levels_p is not None:
            return self.levels_p.shape[1] - 1
        return self.layer_p.shape[1]

    def p_max_atm(self) -> float:
        """Largest layer pressure [atm], forward.py:190 (host copy of the device formula)."""
        if self.layer_p is not None:
            return float(self.layer_p.max()) if self.layer_p.size else 1.0
        p = self.levels_p
        return float((np.sqrt(p[:, :-1] * p[:, 1:]) / P_STD_HPA).max())


@dataclass
class EngineResult:
    od: object = None              # torch tensor [n_prof, n_lay, n_nu] (float32 or float64)
    trans: object = None           # torch float64 [n_prof, n_nu]
    tau: object = None             # torch float64 [n_prof, n_nu]
    channels: object = None        # torch float64 [n_prof, n_ch] channel-mean transmittance
    evals: int = 0                 # Voigt evaluations under the reference tile rule
    work: int = 0                  # Faddeeva evaluations actually performed (multi-level engine)
    work_split: tuple = ()         # (node evaluations, level-3 loop evaluations, near-zone points)
    groups: List[Group] = field(default_factory=list)
    pending: object = None         # the deferred error check of Job.run(defer_errors=True)

    def check(self) -> None:
        """Raise the device error of a run made with ``defer_errors=True`` (waits for that run's
        device work); a no-op for other results and after the first call."""
        if self.pending is not None:
            f, self.pending = self.pending, None
            f()


_GRID_POOL = None


def grid_async(grid: Grid):
    """Future of ``grid.nu`` computed on a worker thread (NumPy releases the GIL), so the
    host builds the returned grid while the device computes."""
    global _GRID_POOL
    if _GRID_POOL is None:
        from concurrent.futures import ThreadPoolExecutor
        _GRID_POOL = ThreadPoolExecutor(max_workers=1, thread_name_prefix="lbl-grid")
    return _GRID_POOL.submit(lambda: grid.nu)


def to_host(t) -> np.ndarray:
    """Device tensor -> NumPy array through a pinned (page-locked) buffer from torch's
    caching host allocator; the returned array owns that buffer."""
    torch = _torch()
    h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
    h.copy_(t, non_blocking=True)
    torch.cuda.current_stream().synchronize()
    return h.numpy()


def _upload(torch, a, dtype, device, non_blocking: bool = False):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=dtype)).to(device, non_blocking=non_blocking)


def sort_launches(n_lines: int) -> int:
    """Kernels enqueued by lbl_sort_lines for n_lines (keys + bitonic stages)."""
    n_pad = 2048
    while n_pad < n_lines:
        n_pad <<= 1
    n, k = 2, 4096
    while k <= n_pad:
        n += (k.bit_length() - 1) - 11 + 1
        k <<= 1
    return n


class Job:
    """Device-resident inputs of one forward call.

    Construction does the host part (group selection with the reference's
    warnings/errors, grid sizes) and uploads lines, levels and partition tables;
    :meth:`run` then does only device work, with no host read-back before the
    results.

    ``line_window = (lo, hi)`` narrows the device sort's band mask (``forward.py:190-220``)
    to [max(nu_first - cutoff, lo), min(nu_last + cutoff, hi)], so only the lines of a
    wavenumber shard are gathered and prepared (its tiles' windows widened by the
    cut-off and the largest pressure shift, as ``shard.line_window`` gives). Every line
    the full job keeps inside that window is kept, in the same order, and group
    selection, warnings and the shift pad still come from the whole line list, so the
    shard's tiles see the same candidate lines as in the full job and their sums are
    identical.
    """

    def __init__(self, sd: SpectralData, layers: LayerInput, grid: Grid, cutoff: float, warn_level: int = 4,
                 line_window: Optional[Tuple[float, float]] = None):
        _lib.load()
        torch = _torch()
        self.torch = torch
        self.dev = torch.device("cuda", torch.cuda.current_device())
        self.grid, self.cutoff, self.layers = grid, float(cutoff), layers
        self.n_prof, self.n_lay = layers.n_prof, layers.n_lay
        self.p_max = layers.p_max_atm() if self.n_lay > 0 else 1.0
        self.nu_first, self.nu_last = grid.nu_at(0), grid.nu_at(grid.n_nu - 1)
        self.h2d_bytes = 0
        # the line arrays go to the device while the host selects the groups
        L = sd.lines
        staged = self._stage_lines(L)
        st = {}
        try:
            self.groups, gid = select_groups(sd, layers.gases, self.nu_first, self.nu_last, self.cutoff,
                                             self.p_max, warn_level + 1, stats=st)
        finally:
            self.lines_in = self._finish_lines(staged)
        self.n_lines = int(gid.size)
        self.mask_lo, self.mask_hi = band_edges(self.nu_first, self.nu_last, self.cutoff, line_window)
        band_lines = int(st["band_lines"])
        if line_window is not None and self.groups:
            c = lambda k: np.ascontiguousarray(L[k], dtype=np.float64)
            nu0, shift = c("nu0"), c("shift")
            band_lines = int(_lib.load_host().lbl_count_band(nu0.ctypes.data, shift.ctypes.data, gid.ctypes.data,
                                                             self.n_lines, self.mask_lo, self.mask_hi,
                                                             float(self.p_max)))
        # device records are sized for this host count (a bound on the sort's kept count),
        # so no stage waits for the device count; slots past the device count are inactive
        self.n_bound = band_lines
        self.empty = not self.groups or self.n_lay == 0 or band_lines <= 0
        if self.empty:
            return
        if self.n_lines > (1 << 30):
            raise ValueError("at most 2^30 lines per call")
        span = (self.nu_last - self.nu_first + 2 * self.cutoff) / grid.step + 2 * grid.n_nu
        if not math.isfinite(span) or span > 1.5e9:
            raise ValueError("grid index range exceeds the engine's 32-bit line index")
        # the small inputs go up together: one page-locked buffer, one copy, typed views
        gas_index = {g: i for i, g in enumerate(layers.gases)}
        offs = np.cumsum([0] + [g.tips_t.size for g in self.groups[:-1]])
        if layers.levels_p is not None:
            lay = [(layers.levels_p, np.float64), (layers.levels_t, np.float64), (layers.levels_vmr, np.float64)]
        else:
            lay = [(layers.layer_p, np.float64), (layers.layer_t, np.float64), (layers.layer_vmr, np.float64),
                   (layers.layer_col, np.float64)]
        grp = [([gas_index[g.gas] for g in self.groups], np.int32), ([g.molar_mass for g in self.groups], np.float64),
               (offs, np.int32), ([g.tips_t.size for g in self.groups], np.int32),
               (np.concatenate([g.tips_t for g in self.groups]), np.float64),
               (np.concatenate([g.tips_q for g in self.groups]), np.float64)]
        views = self._up_packed(lay + grp + [(gid, np.int32)])
        if layers.levels_p is not None:
            self.lv, self.lay = tuple(views[:3]), None
        else:
            self.lv, self.lay = None, tuple(views[:4])
        self.grp = tuple(views[len(lay):len(lay) + 6])
        self.gid = views[-1]
        self.pad = float(st["max_abs_shift"]) * self.p_max * (1 + 1e-9) + 1e-9

    LINE_KEYS = ("nu0", "Sref", "g_air", "g_self", "Elow", "n_air", "shift")

    def _stage_lines(self, L):
        """Start moving the seven float64 line columns to the device. Page-locked columns
        are copied asynchronously right away; pageable ones (ordinary NumPy arrays) are
        packed into one page-locked buffer by a worker thread while the caller's thread
        selects the groups, and :meth:`_finish_lines` then issues one asynchronous copy."""
        torch = self.torch
        arrs = [np.ascontiguousarray(L[k], dtype=np.float64) for k in self.LINE_KEYS]
        n = arrs[0].size
        if n == 0 or any(a.size != n for a in arrs) or all(torch.from_numpy(a).is_pinned() for a in arrs):
            return tuple(self._up(a, np.float64, non_blocking=True) for a in arrs)
        host = torch.empty((len(arrs), n), dtype=torch.float64, pin_memory=True)
        hb = host.numpy()

        def pack():
            for i, a in enumerate(arrs):
                hb[i] = a                    # NumPy copies without holding the GIL

        worker = threading.Thread(target=pack, name="lbl-pack")
        worker.start()
        return host, worker

    def _finish_lines(self, staged):
        if len(staged) == len(self.LINE_KEYS):      # already on its way (page-locked columns)
            return staged
        host, worker = staged
        worker.join()
        dev = host.to(self.dev, non_blocking=True)   # the caching host allocator keeps host alive
        self.h2d_bytes += host.numel() * host.element_size()
        return tuple(dev[i] for i in range(dev.shape[0]))

    def _up(self, a, dtype, non_blocking: bool = False):
        t = _upload(self.torch, a, dtype, self.dev, non_blocking)
        self.h2d_bytes += t.numel() * t.element_size()
        return t

    def _up_packed(self, items):
        """Upload [(array, dtype), ...] through one page-locked buffer and one asynchronous
        copy; returns contiguous device tensors (views of one allocation, 256-B aligned)."""
        torch = self.torch
        arrs = [np.ascontiguousarray(a, dtype=dt) for a, dt in items]
        offs, total = [], 0
        for a in arrs:
            offs.append(total)
            total += -(-max(a.nbytes, 1) // 256) * 256
        host = torch.empty(total, dtype=torch.uint8, pin_memory=True)
        hb = host.numpy()
        for a, o in zip(arrs, offs):
            hb[o:o + a.nbytes] = a.reshape(-1).view(np.uint8)
        dev = torch.empty(total, dtype=torch.uint8, device=self.dev)
        dev.copy_(host, non_blocking=True)        # the caching host allocator keeps host alive until done
        self.h2d_bytes += sum(a.nbytes for a in arrs)
        tdt = {np.dtype(np.float64): torch.float64, np.dtype(np.int32): torch.int32}
        return [dev[o:o + a.nbytes].view(tdt[a.dtype]).reshape(a.shape) for a, o in zip(arrs, offs)]

    def _device_lines(self, stream):
        """Layers, per-(layer, group) records, band mask + sort, gather and tile ranges.

        Returns (t_layer, layer_groups, lines, n_rec, ranges, n_grp): n_rec is the host's
        bound on the kept lines, the record count of every per-line buffer (the device
        count stays on the device).
        """
        torch, dev = self.torch, self.dev
        grid = self.grid
        n_prof, n_lay, n_nu = self.n_prof, self.n_lay, grid.n_nu
        n_rows = n_prof * n_lay
        n_gas = len(self.layers.gases)
        if self.lv is not None:
            lp, lt, lv = self.lv
            p_atm = torch.empty((n_prof, n_lay), dtype=torch.float64, device=dev)
            t_lay = torch.empty_like(p_atm)
            v_lay = torch.empty((n_prof, n_gas, n_lay), dtype=torch.float64, device=dev)
            col = torch.empty_like(v_lay)
            _lib.call("lbl_build_layers", lp.data_ptr(), lt.data_ptr(), lv.data_ptr(), n_prof, n_lay + 1, n_gas,
                      COLUMN_FACTOR, p_atm.data_ptr(), t_lay.data_ptr(), v_lay.data_ptr(), col.data_ptr(),
                      stream)
            self.launches += 1
        else:
            p_atm, t_lay, v_lay, col = self.lay
        # per (layer, group)
        n_grp = len(self.groups)
        grp_gas, grp_mass, tips_off, tips_len, tips_t, tips_q = self.grp
        lg = torch.empty((n_rows * n_grp * _lib.SIZEOF_LAYER_GROUP // 8,), dtype=torch.float64, device=dev)
        _lib.call("lbl_layer_groups", t_lay.data_ptr(), p_atm.data_ptr(), v_lay.data_ptr(), col.data_ptr(),
                  n_prof, n_lay, n_gas, n_grp, grp_gas.data_ptr(), grp_mass.data_ptr(), tips_off.data_ptr(),
                  tips_len.data_ptr(), tips_t.data_ptr(), tips_q.data_ptr(), lg.data_ptr(), stream)
        self.launches += 1
        # lines: mask, sort, gather
        d_nu0, d_sref, d_gair, d_gself, d_elow, d_nair, d_shift = self.lines_in
        n_lines = self.n_lines
        ws_bytes = _lib.load().lbl_sort_workspace_bytes(n_lines)
        ws = torch.empty((ws_bytes + 7) // 8, dtype=torch.float64, device=dev)
        order = torch.empty(n_lines, dtype=torch.int32, device=dev)
        kept = torch.empty(1, dtype=torch.int32, device=dev)
        max_sb = torch.empty(1, dtype=torch.float64, device=dev)
        _lib.call("lbl_sort_lines", d_nu0.data_ptr(), d_shift.data_ptr(), self.gid.data_ptr(), n_lines,
                  self.mask_lo, self.mask_hi, self.p_max, ws.data_ptr(), ws_bytes,
                  order.data_ptr(), kept.data_ptr(), max_sb.data_ptr(), stream)
        self.launches += sort_launches(n_lines)
        self._kept = kept
        n_kept = self.n_bound                          # >= the device's kept count
        lines = torch.empty((n_kept * _lib.SIZEOF_LINE_IN // 8,), dtype=torch.float64, device=dev)
        _lib.call("lbl_gather_lines", d_nu0.data_ptr(), d_sref.data_ptr(), d_gair.data_ptr(), d_gself.data_ptr(),
                  d_elow.data_ptr(), d_nair.data_ptr(), d_shift.data_ptr(), self.gid.data_ptr(), order.data_ptr(),
                  kept.data_ptr(), n_kept, lines.data_ptr(), stream)
        n_tiles = (n_nu + grid.tile_samples - 1) // grid.tile_samples
        ranges = torch.empty((n_tiles, 2), dtype=torch.int32, device=dev)
        _lib.call("lbl_tile_ranges", lines.data_ptr(), kept.data_ptr(), grid.nu_min, grid.step, n_nu,
                  grid.tile_samples, self.cutoff, self.pad, n_tiles, ranges.data_ptr(), stream)
        self.launches += 2
        return t_lay, lg, lines, n_kept, ranges, n_grp

    def _raise_on_error(self, err, n_grp: int) -> None:
        """FloatingPointError for the first failing (layer, group) of the device error word."""
        key = int(err.item())
        if key != INT_MAX:
            row, g = divmod(key, n_grp + 1)
            k = row % self.n_lay
            if g < n_grp:
                raise FloatingPointError(
                    f"Layer {k}, gas '{self.groups[g].gas}': non-finite or negative line strength")
            raise FloatingPointError(f"Layer {k}: non-finite optical depth after radiation term")

    def jacobian(self, gas: str = "H2O", g_tau=None, deterministic: bool = False):
        """Per-layer Jacobians of the float32 multi-level engine.

        Returns device tensors (od, d tau/dT_layer, d tau/dlnVMR_layer of ``gas``),
        each [n_prof, n_lay, n_nu] float32; with ``g_tau`` ([n_prof, n_nu]) returns
        instead the vector-Jacobian products (sum_nu g dtau/dT, sum_nu g dtau/dlnVMR),
        each [n_prof, n_lay] float64, without storing the Jacobian.
        ``deterministic`` selects the bit-reproducible near-zone sums.
        """
        self.launches = 0
        return _jacobian_impl(self, gas, g_tau, deterministic)

    def run(self, precision: str = "fp32", mu: Optional[Sequence[float]] = None, want_od: bool = True,
            want_tau: bool = False, want_trans: bool = False, count_evals: bool = False,
            timer: Optional[dict] = None, channels: Optional[Tuple[int, int]] = None,
            deterministic: bool = False, tiles: Optional[Tuple[int, int]] = None,
            defer_errors: bool = False) -> EngineResult:
        """All device stages; ``timer`` (dict) receives CUDA-event times of the summation kernel.

        The device error word (non-finite or negative line strengths, non-finite optical
        depths) is read at the end, which waits for the device. ``defer_errors=True`` skips
        that wait: the call returns once every stage is queued and ``result.check()`` raises
        the error later, so a caller can queue the next call while this one runs.

        ``channels = (width_points, n_channels)`` adds channel-mean transmittances
        over consecutive half-open blocks of ``width_points`` grid points.
        ``tiles = (first, count)`` (multi-level float32 engine only) computes just those
        reference tiles of the grid: od, tau and trans then cover their points only,
        with the grid values of the full grid (a wavenumber shard).
        """
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {PRECISIONS}, got {precision!r}")
        if deterministic and precision == "fp32-direct":
            raise ValueError("deterministic=True needs precision 'fp32' (multi-level) or 'fp64'")
        torch, dev = self.torch, self.dev
        stream = torch.cuda.current_stream().cuda_stream
        grid = self.grid
        n_prof, n_lay, n_nu = self.n_prof, self.n_lay, grid.n_nu
        n_rows = n_prof * n_lay
        n_tiles = -(-n_nu // grid.tile_samples)
        t_first, t_count = (0, n_tiles) if tiles is None else (int(tiles[0]), int(tiles[1]))
        if tiles is not None:
            if precision != "fp32" or channels is not None:
                raise ValueError("tiles needs precision 'fp32' and no channels")
            if t_first < 0 or t_count < 1 or t_first + t_count > n_tiles:
                raise ValueError(f"tiles ({t_first}, {t_count}) outside the grid's {n_tiles} tiles")
        n_nu = min(n_nu, (t_first + t_count) * grid.tile_samples) - t_first * grid.tile_samples
        res = EngineResult(groups=self.groups)
        single = precision != "fp64"
        od_dtype = torch.float32 if single else torch.float64
        self.launches = 0

        # view cosines go up before any device stage: a pageable copy queued behind the
        # summation would hold the host until the summation ends
        mu_d = None
        if want_tau or want_trans or channels is not None:
            mu_d = torch.as_tensor(np.broadcast_to(np.asarray(1.0 if mu is None else mu, np.float64),
                                                   (n_prof,)).copy()).to(dev)

        def finish(od):
            res.od = od if want_od else None
            if channels is not None:
                width, n_ch = channels
                out = torch.empty((n_prof, n_ch), dtype=torch.float64, device=dev)
                fn = "lbl_channel_mean_f32" if od.dtype == torch.float32 else "lbl_channel_mean_f64"
                _lib.call(fn, od.data_ptr(), n_prof, n_lay, n_nu, mu_d.data_ptr(), 0, int(width), int(n_ch),
                          out.data_ptr(), stream)
                self.launches += 1
                res.channels = out
            if want_tau or want_trans:
                tau = torch.empty((n_prof, n_nu), dtype=torch.float64, device=dev) if want_tau else None
                tr = torch.empty((n_prof, n_nu), dtype=torch.float64, device=dev) if want_trans else None
                fn = "lbl_layer_sum_exp_f32" if od.dtype == torch.float32 else "lbl_layer_sum_exp_f64"
                if timer is not None:
                    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    s0.record()
                _lib.call(fn, _lib.ptr(od), n_prof, n_lay, n_nu, _lib.ptr(mu_d), _lib.ptr(tr), _lib.ptr(tau),
                          stream)
                if timer is not None:
                    s1.record()
                    timer.setdefault("sum_events", []).append((s0, s1))
                self.launches += 1
                res.tau, res.trans = tau, tr
            return res

        if self.empty:
            return finish(torch.zeros((n_prof, n_lay, n_nu), dtype=od_dtype, device=dev))
        st = self._device_lines(stream)
        if st is None:
            return finish(torch.zeros((n_prof, n_lay, n_nu), dtype=od_dtype, device=dev))
        t_lay, lg, lines, n_kept, ranges, n_grp = st
        kept = self._kept
        # per (layer, line) prep and the Voigt sums
        err = torch.full((1,), INT_MAX, dtype=torch.int32, device=dev)
        evals = torch.zeros(4, dtype=torch.int64, device=dev) if count_evals else None
        od = torch.empty((n_prof, n_lay, n_nu), dtype=od_dtype, device=dev)
        rec = _lib.SIZEOF_LINE_F32 if single else _lib.SIZEOF_LINE_F64
        prep = torch.empty((n_rows * n_kept * rec // 8,), dtype=torch.float64, device=dev)
        self.last_prep_bytes = n_rows * n_kept * rec          # prepared line records of the summation
        if precision == "fp32":                               # lines that can be inner lines of a tile's chunks
            inner = torch.empty_like(ranges)
            _lib.call("lbl_ml_inner_ranges", lines.data_ptr(), kept.data_ptr(), grid.nu_min, grid.step,
                      grid.n_nu, grid.tile_samples, self.pad, ranges.shape[0], inner.data_ptr(), stream)
        if timer is not None:
            p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            p0.record()
            timer["prep_shape"] = (n_rows, n_kept, n_grp, rec)
        if single:
            _lib.call("lbl_line_prep_f32", lines.data_ptr(), kept.data_ptr(), n_kept, lg.data_ptr(), n_rows, n_grp,
                      grid.nu_min, grid.step, prep.data_ptr(), err.data_ptr(), stream)
        else:
            _lib.call("lbl_line_prep_f64", lines.data_ptr(), kept.data_ptr(), n_kept, lg.data_ptr(), n_rows, n_grp,
                      prep.data_ptr(), err.data_ptr(), stream)
        if timer is not None:
            p1.record()
            timer.setdefault("prep_events", []).append((p0, p1))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
        common = (prep.data_ptr(), n_kept, ranges.data_ptr(), t_lay.data_ptr(), n_rows, grid.nu_min, grid.step,
                  grid.n_nu, grid.tile_samples, self.cutoff, n_grp, od.data_ptr(), err.data_ptr(),
                  _lib.ptr(evals))
        if precision == "fp32":
            l1_work = torch.empty((_lib.load().lbl_ml_work_floats(n_rows, grid.tile_samples, t_count),),
                                  dtype=torch.float32, device=dev)
            _lib.call("lbl_tau_tiles_ml_f32", common[0], common[1], common[2], inner.data_ptr(), l1_work.data_ptr(),
                      *common[3:], 0 if evals is None else evals.data_ptr() + 8, t_first, t_count,
                      _lib.LBL_DETERMINISTIC if deterministic else 0, stream)
            self.launches += 2
        else:
            _lib.call("lbl_tau_tiles_f32" if single else "lbl_tau_tiles_f64", *common, stream)
        if timer is not None:
            e1.record()
            timer.setdefault("tau_events", []).append((e0, e1))
        self.launches += 2
        finish(od)                          # queue the layer sums before the error word is read
        if defer_errors and evals is None:
            res.pending = lambda: self._raise_on_error(err, n_grp)
        else:
            self._raise_on_error(err, n_grp)
        if evals is not None:
            ev = evals.cpu().tolist()
            res.evals = int(ev[0])
            if precision == "fp32":
                res.work_split = tuple(int(v) for v in ev[1:4])
                res.work = sum(res.work_split)
            else:
                res.work = int(ev[0])
        return res


def _jacobian_impl(job: Job, gas: str, g_tau=None, deterministic: bool = False):
    """Device stages of Job.jacobian."""
    torch, dev = job.torch, job.dev
    stream = torch.cuda.current_stream().cuda_stream
    grid = job.grid
    n_prof, n_lay, n_nu = job.n_prof, job.n_lay, grid.n_nu
    n_rows = n_prof * n_lay

    def zeros():
        if g_tau is not None:
            z = torch.zeros((n_prof, n_lay), dtype=torch.float64, device=dev)
            return z, z.clone()
        z = torch.zeros((n_prof, n_lay, n_nu), dtype=torch.float32, device=dev)
        return z, z.clone(), z.clone()

    if job.empty:
        return zeros()
    st = job._device_lines(stream)
    if st is None:
        return zeros()
    t_lay, lg, lines, n_kept, ranges, n_grp = st
    err = torch.full((1,), INT_MAX, dtype=torch.int32, device=dev)
    prep = torch.empty((n_rows * n_kept * _lib.SIZEOF_LINE_F32 // 8,), dtype=torch.float64, device=dev)
    _lib.call("lbl_line_prep_f32", lines.data_ptr(), job._kept.data_ptr(), n_kept, lg.data_ptr(), n_rows, n_grp,
              grid.nu_min, grid.step, prep.data_ptr(), err.data_ptr(), stream)
    mask = 0
    for i, grp in enumerate(job.groups):
        if grp.gas == gas:
            mask |= 1 << i
    _, _, tips_off, tips_len, tips_t, tips_q = job.grp
    dlnq = torch.empty((n_rows * n_grp,), dtype=torch.float64, device=dev)
    jprep = torch.empty((n_rows * n_kept * _lib.SIZEOF_LINE_JAC // 8,), dtype=torch.float64, device=dev)
    _lib.call("lbl_line_prep_jac", lines.data_ptr(), n_kept, lg.data_ptr(), n_rows, n_grp, tips_off.data_ptr(),
              tips_len.data_ptr(), tips_t.data_ptr(), tips_q.data_ptr(), mask, dlnq.data_ptr(), jprep.data_ptr(),
              stream)
    job.launches += 4
    flags = _lib.LBL_DETERMINISTIC if deterministic else 0
    # inner-line ranges of the forward's chunks: a superset for the Jacobian's smaller chunks
    inner = torch.empty_like(ranges)
    _lib.call("lbl_ml_inner_ranges", lines.data_ptr(), job._kept.data_ptr(), grid.nu_min, grid.step, n_nu,
              grid.tile_samples, job.pad, ranges.shape[0], inner.data_ptr(), stream)
    near = torch.empty_like(ranges)         # level-1 lines within four chunk half-widths
    _lib.call("lbl_jac_near_ranges", lines.data_ptr(), job._kept.data_ptr(), grid.nu_min, grid.step, n_nu,
              grid.tile_samples, job.pad, ranges.shape[0], near.data_ptr(), stream)
    l1_work = torch.empty((_lib.load().lbl_jacobian_ml_work_floats(n_rows, n_nu, grid.tile_samples),),
                          dtype=torch.float32, device=dev)
    job.launches += 3                       # the two range searches and the Jacobian's level-1 kernel
    common = (prep.data_ptr(), jprep.data_ptr(), n_kept, ranges.data_ptr(), inner.data_ptr(), near.data_ptr(),
              t_lay.data_ptr(), n_rows, n_lay, grid.nu_min, grid.step, n_nu, grid.tile_samples, job.cutoff,
              l1_work.data_ptr())
    if g_tau is not None:
        g = torch.as_tensor(g_tau).to(device=dev, dtype=torch.float64).reshape(n_prof, n_nu).contiguous()
        vt = torch.zeros((n_prof, n_lay), dtype=torch.float64, device=dev)
        vv = torch.zeros_like(vt)
        _lib.call("lbl_jacobian_ml_f32", *common, 0, 0, 0, g.data_ptr(), vt.data_ptr(), vv.data_ptr(), flags,
                  stream)
        job._raise_on_error(err, n_grp)          # the line-strength check, read once at the end
        return vt, vv
    od = torch.empty((n_prof, n_lay, n_nu), dtype=torch.float32, device=dev)
    d_t = torch.empty_like(od)
    d_v = torch.empty_like(od)
    _lib.call("lbl_jacobian_ml_f32", *common, od.data_ptr(), d_t.data_ptr(), d_v.data_ptr(), 0, 0, 0, flags, stream)
    job._raise_on_error(err, n_grp)              # the line-strength check, read once at the end
    return od, d_t, d_v


def optical_depth(sd: SpectralData, layers: LayerInput, grid: Grid, cutoff: float,
                  precision: str = "fp32", mu: Optional[Sequence[float]] = None,
                  want_od: bool = True, want_tau: bool = False, want_trans: bool = False,
                  warn_level: int = 4, count_evals: bool = False, deterministic: bool = False) -> EngineResult:
    """Upload one forward call and run every device stage (see the module docstring)."""
    if precision not in PRECISIONS:
        raise ValueError(f"precision must be one of {PRECISIONS}, got {precision!r}")
    job = Job(sd, layers, grid, cutoff, warn_level + 1)
    return job.run(precision, mu, want_od, want_tau, want_trans, count_evals, deterministic=deterministic)


def layer_input_from_profile(profile) -> LayerInput:
    """Levels of one AtmosphericProfile (layers are built on the device)."""
    gases = list(profile.vmr.keys())
    vmr = np.stack([profile.vmr[g] for g in gases])[None] if gases else np.zeros((1, 0, profile.n_levels))
    return LayerInput(gases=gases, levels_p=profile.pressure_hpa[None, :], levels_t=profile.temperature_k[None, :],
                      levels_vmr=vmr)


def layer_input_from_layers(layers) -> LayerInput:
    """Host-built layers (the reference's _Layers object)."""
    gases = list(layers.column_cm2.keys())
    n = layers.n_layers
    vmr = np.stack([layers.vmr[g] for g in gases])[None] if gases else np.zeros((1, 0, n))
    col = np.stack([layers.column_cm2[g] for g in gases])[None] if gases else np.zeros((1, 0, n))
    return LayerInput(gases=gases, layer_p=np.asarray(layers.pressure_atm, np.float64)[None, :],
                      layer_t=np.asarray(layers.temperature_k, np.float64)[None, :],
                      layer_vmr=vmr, layer_col=col)
