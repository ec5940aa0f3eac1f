"""ctypes access to the CPU checkers.

TEST INFRASTRUCTURE ONLY. Imported by tests/, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py``; the product package never imports it.

Two checkers share one interface:

* ``Oracle("port")``      -- oracle/liboracle_pv.so, the C restatement (pv_oracle.c);
* ``Oracle("reference")`` -- oracle/_ref/libpvref.so, the unmodified reference compiled from its
  own sources (oracle/Makefile, target ``ref``) behind ref_shim.cpp.

Both raise the Python analogue of the reference's exception type: ValueError for
std::invalid_argument, IndexError for std::out_of_range, RuntimeError for std::runtime_error.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "liboracle_pv.so")
REF_LIB = os.path.join(HERE, "_ref", "libpvref.so")
REF_CUDA_LIB = os.path.join(HERE, "_ref", "libpvref_cuda.so")
REF_DIR = os.path.join(HERE, "_ref")

GEOMETRIES = {"infinite": 0, "periodic": 1, "disk": 2}


class _Params(ctypes.Structure):
    _fields_ = [
        ("geometry", ctypes.c_int),
        ("core_radius", ctypes.c_double),
        ("box_length_x", ctypes.c_double),
        ("box_length_y", ctypes.c_double),
        ("image_layers", ctypes.c_int),
        ("disk_radius", ctypes.c_double),
        ("absolute_tolerance", ctypes.c_double),
        ("relative_tolerance", ctypes.c_double),
        ("minimum_time_step", ctypes.c_double),
        ("maximum_time_step", ctypes.c_double),
        ("dipole_removal", ctypes.c_int),
        ("dipole_removal_distance", ctypes.c_double),
        ("dipole_reinjection", ctypes.c_int),
        ("random_seed", ctypes.c_uint64),
    ]


class _Candidate(ctypes.Structure):
    _fields_ = [("first", ctypes.c_size_t), ("second", ctypes.c_size_t),
                ("distance_squared", ctypes.c_double)]


@dataclass
class Geometry:
    """Parameters of one simulation (the fields of the reference's SimParams that the hot path
    reads; defaults follow src/params.h:37-78)."""

    boundary: str = "infinite"
    core_radius: float = 0.0
    box_length_x: float = 2.0
    box_length_y: float = 2.0
    image_layers: int = 8
    disk_radius: float = 1.0
    absolute_tolerance: float = 1e-10
    relative_tolerance: float = 1e-8
    minimum_time_step: float = 1e-12
    maximum_time_step: float = 0.1
    dipole_removal: bool = False
    dipole_removal_distance: float = 0.01
    dipole_reinjection: int = 0
    random_seed: int = 1234567

    def c(self) -> _Params:
        return _Params(GEOMETRIES[self.boundary], self.core_radius, self.box_length_x,
                       self.box_length_y, self.image_layers, self.disk_radius,
                       self.absolute_tolerance, self.relative_tolerance, self.minimum_time_step,
                       self.maximum_time_step, int(self.dipole_removal),
                       self.dipole_removal_distance, self.dipole_reinjection, self.random_seed)


_EXC = {1: ValueError, 2: IndexError, 3: RuntimeError, 4: NotImplementedError, 9: RuntimeError}
_D = ctypes.POINTER(ctypes.c_double)


def _p(a: np.ndarray):
    return a.ctypes.data_as(_D)


def build(reference: bool = False) -> None:
    """Compile the checker(s) with oracle/Makefile (the reference only where its sources are)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    if reference:
        subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)


class Oracle:
    """One CPU checker. ``kind`` is "port" (the C restatement) or "reference"."""

    def __init__(self, kind: str = "port"):
        self.kind = kind
        path = PORT_LIB if kind == "port" else REF_LIB
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is missing; run make -C oracle{' ref' if kind != 'port' else ''}")
        lib = ctypes.CDLL(path)
        self.lib = lib
        pre = "pvo_" if kind == "port" else "pvref_"
        self._pre = pre
        getattr(lib, pre + "last_error").restype = ctypes.c_char_p
        sz = ctypes.c_size_t
        P = ctypes.POINTER(_Params)
        getattr(lib, pre + "evaluate_range").argtypes = [P, _D, _D, _D, sz, sz, sz, _D, _D]
        getattr(lib, pre + "hamiltonian").argtypes = [P, _D, _D, _D, sz, _D]
        getattr(lib, pre + "invariants").argtypes = [P, _D, _D, _D, sz, _D]
        getattr(lib, pre + "stepper_create").argtypes = [P, sz]
        getattr(lib, pre + "stepper_create").restype = ctypes.c_void_p
        getattr(lib, pre + "stepper_destroy").argtypes = [ctypes.c_void_p]
        getattr(lib, pre + "stepper_invalidate").argtypes = [ctypes.c_void_p]
        if kind == "port":
            lib.pvo_evaluate.argtypes = [P, _D, _D, _D, sz, _D, _D]
            lib.pvo_rk4_step.argtypes = [ctypes.c_void_p, _D, _D, _D, sz, ctypes.c_double]
            lib.pvo_dopri5_step.argtypes = [ctypes.c_void_p, _D, _D, _D, sz, ctypes.c_double, _D]
            lib.pvo_stepper_evaluations.argtypes = [ctypes.c_void_p]
            lib.pvo_stepper_evaluations.restype = sz
            lib.pvo_dipole_scan.argtypes = [P, _D, _D, _D, sz, ctypes.POINTER(_Candidate), sz,
                                            ctypes.POINTER(sz)]
        else:
            lib.pvref_rk4_steps.argtypes = [ctypes.c_void_p, _D, _D, _D, sz, ctypes.c_double, sz]
            lib.pvref_dopri5_step.argtypes = [ctypes.c_void_p, _D, _D, _D, sz, ctypes.c_double, _D]
            lib.pvref_dipole_process.argtypes = [P, _D, _D, _D, ctypes.POINTER(sz), sz,
                                                 ctypes.POINTER(sz)]
            lib.pvref_dipole_process_state.argtypes = [
                P, _D, _D, _D, ctypes.POINTER(sz), sz, ctypes.POINTER(sz),
                ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64), ctypes.c_char_p,
                ctypes.c_char_p, sz]
            lib.pvref_max_threads.restype = ctypes.c_int
            lib.pvref_set_threads.argtypes = [ctypes.c_int]

    def _check(self, rc: int) -> None:
        if rc:
            msg = getattr(self.lib, self._pre + "last_error")().decode()
            raise _EXC.get(rc, RuntimeError)(msg)

    @staticmethod
    def _arrays(x, y, g):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.ascontiguousarray(y, dtype=np.float64)
        g = np.ascontiguousarray(g, dtype=np.float64)
        if not (x.shape == y.shape == g.shape):
            raise ValueError("vortex arrays have different lengths")
        return x, y, g

    def evaluate(self, geo: Geometry, x, y, g):
        """VelocityKernel::evaluate (src/compute.cpp:60-69): full range + finiteness check."""
        x, y, g = self._arrays(x, y, g)
        n = x.size
        u = np.empty(n)
        v = np.empty(n)
        par = geo.c()
        if self.kind == "port":
            self._check(self.lib.pvo_evaluate(ctypes.byref(par), _p(x), _p(y), _p(g), n, _p(u), _p(v)))
        else:
            self._check(self.lib.pvref_evaluate_range(ctypes.byref(par), _p(x), _p(y), _p(g), n, 0, n,
                                                      _p(u), _p(v)))
        return u, v

    def evaluate_range(self, geo: Geometry, x, y, g, begin: int, end: int):
        """VelocityKernel::evaluateRange (src/compute.h:26-28); returns u, v for [begin, end)."""
        x, y, g = self._arrays(x, y, g)
        k = max(end - begin, 0)
        u = np.empty(max(k, 1))
        v = np.empty(max(k, 1))
        par = geo.c()
        self._check(getattr(self.lib, self._pre + "evaluate_range")(ctypes.byref(par), _p(x), _p(y), _p(g),
                                                           x.size, begin, end, _p(u), _p(v)))
        return u[:k], v[:k]

    def hamiltonian(self, geo: Geometry, x, y, g) -> float:
        x, y, g = self._arrays(x, y, g)
        out = np.zeros(1)
        par = geo.c()
        self._check(getattr(self.lib, self._pre + "hamiltonian")(ctypes.byref(par), _p(x), _p(y), _p(g),
                                                        x.size, _p(out)))
        return float(out[0])

    def invariants(self, geo: Geometry, x, y, g) -> np.ndarray:
        """computeInvariants: [circulation, Ix, Iy, angular impulse, Hamiltonian]."""
        x, y, g = self._arrays(x, y, g)
        out = np.zeros(5)
        par = geo.c()
        self._check(getattr(self.lib, self._pre + "invariants")(ctypes.byref(par), _p(x), _p(y), _p(g),
                                                       x.size, _p(out)))
        return out

    def stepper(self, geo: Geometry, n: int) -> "Stepper":
        return Stepper(self, geo, n)

    def dipole_scan(self, geo: Geometry, x, y, g):
        """Candidate list of DipoleManager::process (src/dipole.cpp:49-78), in scan order, as an
        (k, 3) array of (first, second, distance^2); second == n marks a disk wall image."""
        if self.kind != "port":
            raise NotImplementedError("the reference exposes the scan only inside process()")
        x, y, g = self._arrays(x, y, g)
        par = geo.c()
        count = ctypes.c_size_t(0)
        cap = 1024
        while True:
            buf = (_Candidate * cap)()
            self._check(self.lib.pvo_dipole_scan(ctypes.byref(par), _p(x), _p(y), _p(g), x.size,
                                                 buf, cap, ctypes.byref(count)))
            if count.value <= cap:
                break
            cap = count.value
        return [(buf[i].first, buf[i].second, buf[i].distance_squared) for i in range(count.value)]

    def dipole_process(self, geo: Geometry, x, y, g):
        """DipoleManager::process on a fresh manager; returns (events, x, y, g) (reference only)."""
        if self.kind == "port":
            raise NotImplementedError("selection and reinjection are host logic of the reference")
        x, y, g = (np.array(a, dtype=np.float64) for a in (x, y, g))
        n = ctypes.c_size_t(x.size)
        cap = x.size
        xx, yy, gg = (np.resize(a, max(cap, 1)).copy() for a in (x, y, g))
        events = ctypes.c_size_t(0)
        par = geo.c()
        self._check(self.lib.pvref_dipole_process(ctypes.byref(par), _p(xx), _p(yy), _p(gg),
                                                  ctypes.byref(n), cap, ctypes.byref(events)))
        k = n.value
        return events.value, xx[:k].copy(), yy[:k].copy(), gg[:k].copy()

    def dipole_events(self, geo: Geometry, x, y, g, state=None):
        """One DipoleManager::process call (src/dipole.cpp:42-127) by a manager restored from
        state = (removed, reinjected, engine text) (src/dipole.cpp:32-40; None: fresh seeding).
        Returns (events, x, y, g, state after the call). The port restates the selection and the
        reinjection draws in Python (DipolePort); the reference runs its own DipoleManager."""
        if self.kind == "port":
            return DipolePort(self, geo, state).process(x, y, g)
        x, y, g = (np.array(a, dtype=np.float64) for a in (x, y, g))
        cap = x.size + 2
        xx, yy, gg = (np.resize(a, max(cap, 1)).copy() for a in (x, y, g))
        n = ctypes.c_size_t(x.size)
        events = ctypes.c_size_t(0)
        removed = ctypes.c_uint64(state[0] if state else 0)
        reinjected = ctypes.c_uint64(state[1] if state else 0)
        out = ctypes.create_string_buffer(1 << 15)
        par = geo.c()
        self._check(self.lib.pvref_dipole_process_state(
            ctypes.byref(par), _p(xx), _p(yy), _p(gg), ctypes.byref(n), cap, ctypes.byref(events),
            ctypes.byref(removed), ctypes.byref(reinjected),
            (state[2] if state else "").encode(), out, len(out)))
        k = n.value
        return (events.value, xx[:k].copy(), yy[:k].copy(), gg[:k].copy(),
                (removed.value, reinjected.value, out.value.decode()))

    def write_trajectory(self, path: str, time: float, frame: int, x, y, g, u, v) -> bytes:
        """TrajectoryWriter (src/print.cpp:24-40): header + one frame, written by the reference
        into `path`; returns the file's bytes (reference only)."""
        if self.kind == "port":
            raise NotImplementedError("the reference's writer is its own ostream code")
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, g, u, v)]
        self.lib.pvref_write_trajectory.argtypes = [ctypes.c_char_p, ctypes.c_double,
                                                    ctypes.c_size_t] + [_D] * 5 + [ctypes.c_size_t]
        self._check(self.lib.pvref_write_trajectory(path.encode(), time, frame,
                                                    *[_p(a) for a in arrs], arrs[0].size))
        with open(path, "rb") as f:
            return f.read()

    def write_checkpoint(self, directory: str, geo: Geometry, x, y, g, initial, segment,
                         dipole_state, schedule, progress) -> bytes:
        """writeCheckpoint (src/checkpoint.cpp:23-102) by the reference; returns the bytes of
        checkpoint_<outputIndex>.dat. dipole_state = (removed, reinjected, engine text);
        schedule = the 5 OutputSchedule fields; progress = (time, suggestedTimeStep,
        nextOutputTime, acceptedSteps, outputIndex, eventIndex)."""
        if self.kind == "port":
            raise NotImplementedError("the reference's writer is its own ostream code")
        x, y, g = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, g))
        inv = np.array(initial, dtype=np.float64)
        seg = np.array(segment, dtype=np.float64)
        sched = np.array(schedule, dtype=np.float64)
        pd = np.array(progress[:3], dtype=np.float64)
        pi = np.array(progress[3:], dtype=np.uint64)
        u64p = ctypes.POINTER(ctypes.c_uint64)
        self.lib.pvref_write_checkpoint.argtypes = [
            ctypes.c_char_p, ctypes.POINTER(_Params), _D, _D, _D, ctypes.c_size_t, _D, _D,
            ctypes.c_uint64, ctypes.c_uint64, ctypes.c_char_p, _D, _D, u64p]
        par = geo.c()
        self._check(self.lib.pvref_write_checkpoint(
            directory.encode(), ctypes.byref(par), _p(x), _p(y), _p(g), x.size, _p(inv), _p(seg),
            int(dipole_state[0]), int(dipole_state[1]), dipole_state[2].encode(), _p(sched),
            _p(pd), pi.ctypes.data_as(u64p)))
        path = os.path.join(directory, "checkpoint_%08d.dat" % int(progress[4]))
        with open(path, "rb") as f:
            return f.read()

    def set_threads(self, n: int) -> None:
        if self.kind != "port":
            self.lib.pvref_set_threads(n)

    def max_threads(self) -> int:
        return self.lib.pvref_max_threads() if self.kind != "port" else 1


class Stepper:
    """RungeKuttaIntegrator (src/timestep.h:18-34) of one checker; keeps the FSAL derivative."""

    def __init__(self, oracle: Oracle, geo: Geometry, n: int):
        self.o = oracle
        self.geo = geo
        self._par = geo.c()
        self.h = getattr(oracle.lib, oracle._pre + "stepper_create")(ctypes.byref(self._par), n)
        if not self.h:
            oracle._check(1)

    def __del__(self):
        if getattr(self, "h", None):
            getattr(self.o.lib, self.o._pre + "stepper_destroy")(self.h)
            self.h = None

    def invalidate(self) -> None:
        getattr(self.o.lib, self.o._pre + "stepper_invalidate")(self.h)

    def rk4_step(self, x, y, g, dt: float):
        x, y, g = (np.array(a, dtype=np.float64) for a in (x, y, g))
        if self.o.kind == "port":
            self.o._check(self.o.lib.pvo_rk4_step(self.h, _p(x), _p(y), _p(g), x.size, dt))
        else:
            self.o._check(self.o.lib.pvref_rk4_steps(self.h, _p(x), _p(y), _p(g), x.size, dt, 1))
        return x, y

    def dopri5_step(self, x, y, g, dt: float):
        """Returns (x, y, [accepted dt, suggested dt, error, rejected])."""
        x, y, g = (np.array(a, dtype=np.float64) for a in (x, y, g))
        out = np.zeros(4)
        fn = self.o.lib.pvo_dopri5_step if self.o.kind == "port" else self.o.lib.pvref_dopri5_step
        self.o._check(fn(self.h, _p(x), _p(y), _p(g), x.size, dt, _p(out)))
        return x, y, out

    @property
    def evaluations(self) -> int:
        if self.o.kind != "port":
            raise NotImplementedError
        return int(self.o.lib.pvo_stepper_evaluations(self.h))


# ---- DipoleManager restated (src/dipole.cpp:29-186) ---------------------------------------------

class MT19937_64:
    """std::mt19937_64: the 64-bit Mersenne Twister of Matsumoto and Nishimura with the
    parameters the C++ standard fixes ([rand.predef]), and libstdc++'s text form of its state
    (the 312 words, then the position, separated by spaces)."""

    N, M = 312, 156
    MATRIX = 0xB5026F5AA96619E9
    UPPER, LOWER = 0xFFFFFFFF80000000, 0x7FFFFFFF
    MASK = (1 << 64) - 1

    def __init__(self, seed: int = 5489):
        mt = [seed & self.MASK]
        for i in range(1, self.N):
            mt.append((6364136223846793005 * (mt[-1] ^ (mt[-1] >> 62)) + i) & self.MASK)
        self.mt, self.p = mt, self.N

    def _twist(self):
        mt, n, m = self.mt, self.N, self.M
        for i in range(n):
            y = (mt[i] & self.UPPER) | (mt[(i + 1) % n] & self.LOWER)
            mt[i] = mt[(i + m) % n] ^ (y >> 1) ^ (self.MATRIX if y & 1 else 0)
        self.p = 0

    def __call__(self) -> int:
        if self.p >= self.N:
            self._twist()
        z = self.mt[self.p]
        self.p += 1
        z ^= (z >> 29) & 0x5555555555555555
        z ^= (z << 17) & 0x71D67FFFEDA60000
        z ^= (z << 37) & 0xFFF7EEE000000000
        z ^= z >> 43
        return z & self.MASK

    def unit(self) -> float:
        """uniform_real_distribution<double>(0, 1): libstdc++'s generate_canonical with one
        64-bit draw -- the draw rounded to double, divided by 2^64, kept below 1."""
        r = float(self()) / 18446744073709551616.0
        return r if r < 1.0 else math.nextafter(1.0, 0.0)

    def text(self) -> str:
        return " ".join(str(w) for w in self.mt) + " " + str(self.p)

    @classmethod
    def from_text(cls, text: str) -> "MT19937_64":
        words = [int(w) for w in text.split()]
        if len(words) != cls.N + 1:
            raise RuntimeError("invalid random-generator state in checkpoint")
        e = cls(0)
        e.mt, e.p = words[:cls.N], words[cls.N]
        return e


class DipolePort:
    """DipoleManager (src/dipole.h:18-40) restated: the candidate scan is the C port's
    (pvo_dipole_scan, bit-exact to src/dipole.cpp:49-78); the closest-first disjoint selection
    (:79-100), the order-keeping compaction (:104-113) and the reinjection draws (:116-180)
    follow here in the reference's order and arithmetic (Python's math functions are the C
    library's)."""

    SEED_MIX = 0xD1B54A32D192ED03     # src/dipole.cpp:29-30

    def __init__(self, oracle: "Oracle", geo: Geometry, state=None):
        self.oracle, self.geo = oracle, geo
        self.removed, self.reinjected = (state[0], state[1]) if state else (0, 0)
        if state and state[2]:
            self.random = MT19937_64.from_text(state[2])
        else:
            self.random = MT19937_64(geo.random_seed ^ self.SEED_MIX)

    def _position(self):
        geo = self.geo
        if geo.boundary == "periodic":
            px = (self.random.unit() - 0.5) * geo.box_length_x
            py = (self.random.unit() - 0.5) * geo.box_length_y
            return px, py
        radius = geo.disk_radius * math.sqrt(self.random.unit())
        angle = 2.0 * math.pi * self.random.unit()
        return radius * math.cos(angle), radius * math.sin(angle)

    def _pair(self, population: int):
        geo = self.geo
        periodic = geo.boundary == "periodic"
        area = (geo.box_length_x * geo.box_length_y if periodic
                else math.pi * geo.disk_radius * geo.disk_radius)
        spacing = math.sqrt(area / float(population))
        first = self._position()
        second = self._position()
        if geo.dipole_reinjection == 2:
            for _ in range(100000):
                first = self._position()
                angle = 2.0 * math.pi * self.random.unit()
                second = (first[0] + spacing * math.cos(angle), first[1] + spacing * math.sin(angle))
                if periodic:
                    second = (math.remainder(second[0], geo.box_length_x),
                              math.remainder(second[1], geo.box_length_y))
                    break
                if second[0] * second[0] + second[1] * second[1] < geo.disk_radius * geo.disk_radius:
                    break
            else:
                raise RuntimeError("could not find a valid paired reinjection position")
        return first, second

    def process(self, x, y, g):
        x, y, g = (np.array(a, dtype=np.float64) for a in (x, y, g))
        n = x.size
        geo = self.geo
        if not geo.dipole_removal or n == 0:
            return 0, x, y, g, self.state()
        cands = sorted(self.oracle.dipole_scan(geo, x, y, g), key=lambda c: (c[2], c[0], c[1]))
        selected = np.zeros(n, bool)
        events = []
        for a, b, _ in cands:
            if selected[a] or (b < n and selected[b]):
                continue
            selected[a] = True
            if b < n:
                selected[b] = True
                events.append((g[a], g[b], False))
            else:
                events.append((g[a], 0.0, True))
        if not events:
            return 0, x, y, g, self.state()
        keep = ~selected
        ox, oy, og = list(x[keep]), list(y[keep]), list(g[keep])
        self.removed += len(events)
        if geo.dipole_reinjection != 0:
            for g1, g2, wall in events:
                if wall:
                    radius = geo.disk_radius * math.sqrt(self.random.unit())
                    angle = 2.0 * math.pi * self.random.unit()
                    ox.append(radius * math.cos(angle))
                    oy.append(radius * math.sin(angle))
                    og.append(g1)
                    continue
                first, second = self._pair(n)
                ox += [first[0], second[0]]
                oy += [first[1], second[1]]
                og += [g1, g2]
            self.reinjected += len(events)
        return len(events), np.array(ox), np.array(oy), np.array(og), self.state()

    def state(self):
        return self.removed, self.reinjected, self.random.text()
