"""mechanica_b200: the force-and-step hot path of Mechanica's mdcore engine on a B200.

The Python surface keeps the reference's names, arguments and defaults
(src/MxSimulator.cpp:196-275 for ``init``, src/MxUniverse.cpp:93-108 for the
defaults, src/mdcore/src/MxPotential.cpp:2459-2750 for the potential
factories, src/mdcore/src/bond.cpp:535-560 for ``Bond``):

    import mechanica_b200 as m
    m.init(dim=[10, 10, 10], cells=[10, 10, 10], cutoff=1.0, dt=0.01)
    class Argon(m.Particle):
        mass = 39.4
        radius = 0.1
    pot = m.Potential.lennard_jones_12_6(0.275, 1.0, 9.5075e-6, 6.1545e-3, 1e-3)
    m.bind(pot, Argon, Argon)
    Argon.factory(positions=x, velocities=v)     # or Argon(position, velocity)
    m.Universe.step()

Everything below the Python layer is the C ABI of libmxg.so (include/mxg.h);
all force, bond and integration work runs in CUDA kernels on the device.
"""
import atexit
import ctypes
import math
import weakref

import numpy as np

from . import _native
from ._native import EngineError, check, f32, f64, i32, lib, ptr

__all__ = [
    "init", "Universe", "universe", "Particle", "Potential", "Bond", "Angle", "Dihedral", "Cuboid", "flux", "fick", "secrete", "uptake", "bind", "forces", "step", "run",
    "Newtonian", "Overdamped", "FORWARD_EULER", "RUNGE_KUTTA_4", "BOUNDARY_NONE", "PERIODIC_X", "PERIODIC_Y", "PERIODIC_Z",
    "PERIODIC_FULL", "FREESLIP_X", "FREESLIP_Y", "FREESLIP_Z", "FREESLIP_FULL", "EngineError", "ParticleList",
]

# particle dynamics (src/mdcore/include/MxParticle.h:48-49)
Newtonian = 0
Overdamped = 1
FORWARD_EULER = 0
RUNGE_KUTTA_4 = 1

# integer boundary flags (src/mdcore/include/space.h:44-59)
BOUNDARY_NONE = 0
PERIODIC_X = 1 << 0
PERIODIC_Y = 1 << 1
PERIODIC_Z = 1 << 2
PERIODIC_FULL = PERIODIC_X | PERIODIC_Y | PERIODIC_Z
FREESLIP_X = 1 << 6
FREESLIP_Y = 1 << 7
FREESLIP_Z = 1 << 8
FREESLIP_FULL = FREESLIP_X | FREESLIP_Y | FREESLIP_Z

_BC_VELOCITY, _BC_PERIODIC, _BC_FREESLIP, _BC_POTENTIAL, _BC_NOSLIP = 1, 2, 4, 8, 16
_FACES = ["left", "right", "front", "back", "bottom", "top"]
_AXIS_FACES = {"x": (0, 1), "y": (2, 3), "z": (4, 5)}


def _bc_kind_of(value):
    s = str(value).upper()
    if s == "PERIODIC":
        return _BC_PERIODIC
    if s in ("FREE_SLIP", "FREESLIP"):
        return _BC_FREESLIP
    if s in ("NO_SLIP", "NOSLIP"):
        return _BC_NOSLIP
    if s == "POTENTIAL":
        return _BC_FREESLIP | _BC_POTENTIAL  # a free-slip wall that potentials are usually bound to
    raise ValueError(f"invalid boundary condition {value!r}")


def parse_bc(bc):
    """Maps the reference's ``bc`` argument (MxBoundaryConditions.cpp:501-700) to
    per-face kinds, wall velocities and restitution."""
    kind = [_BC_PERIODIC] * 6
    vel = np.zeros((6, 3), dtype=np.float32)
    restore = np.ones(6, dtype=np.float32)
    if bc is None:
        return kind, vel, restore
    if isinstance(bc, (int, np.integer)):
        kind = [0] * 6
        for axis, bit_p, bit_f in (("x", PERIODIC_X, FREESLIP_X), ("y", PERIODIC_Y, FREESLIP_Y),
                                   ("z", PERIODIC_Z, FREESLIP_Z)):
            k = _BC_PERIODIC if bc & bit_p else (_BC_FREESLIP if bc & bit_f else 0)
            for f in _AXIS_FACES[axis]:
                kind[f] = k
        return kind, vel, restore
    if isinstance(bc, dict):
        kind = [0] * 6
        for axis, faces in _AXIS_FACES.items():
            if axis in bc:
                v = bc[axis]
                vals = v if isinstance(v, (list, tuple)) else [v]
                k = 0
                for item in vals:
                    k |= _bc_kind_of(item)
                for f in faces:
                    kind[f] = k
        for f, name in enumerate(_FACES):
            if name in bc:
                item = bc[name]
                if isinstance(item, dict):
                    kind[f] = _BC_VELOCITY
                    vel[f] = np.asarray(item["velocity"], dtype=np.float32)
                    if "restore" in item:
                        restore[f] = float(item["restore"])
                else:
                    kind[f] = _bc_kind_of(item)
        return kind, vel, restore
    raise TypeError("bc must be an int flag set or a dict")


class PotentialSum:
    """Two potentials summed on the same type pairs (Potential.__add__)."""

    def __init__(self, first, second):
        self.terms = (first, second)
        self.name = f"{first.name} + {second.name}"


class Potential:
    """A tabulated (or DPD) pair potential; factories mirror MxPotential.cpp:2459-2750."""

    def __init__(self, handle, name):
        self._h = ctypes.c_void_p(handle)
        self.name = name

    def __del__(self):
        try:
            if self._h:
                lib().mxg_potential_free(self._h)
        except Exception:
            pass

    @staticmethod
    def _make(fn, args, name):
        h = ctypes.c_void_p()
        check(getattr(lib(), fn)(*args, ctypes.byref(h)), fn)
        return Potential(h.value, name)

    @staticmethod
    def lennard_jones_12_6(min, max, A, B, tol=None):
        tol = 0.001 * (max - min) if tol is None else tol
        return Potential._make("mxg_potential_create_lj126", (min, max, A, B, tol), "Lennard-Jones")

    @staticmethod
    def morse(d=1.0, a=6.0, r0=0.0, min=0.0001, max=3.0, tol=0.001):
        return Potential._make("mxg_potential_create_morse", (d, a, r0, min, max, tol), "Morse")

    @staticmethod
    def harmonic(k, r0, min=None, max=None, tol=None):
        rng = r0
        min = r0 - rng if min is None else min
        max = r0 + rng if max is None else max
        tol = 0.01 * (max - min) if tol is None else tol
        return Potential._make("mxg_potential_create_harmonic", (k, r0, min, max, tol), "Harmonic")

    @staticmethod
    def harmonic_angle(k, theta0, min=0.0, max=math.pi, tol=None):
        """k (theta - theta0)^2, tabulated in cos(theta) (MxPotential.cpp:2577-2590)."""
        tol = 0.005 * abs(max - min) if tol is None else tol
        return Potential._make("mxg_potential_create_harmonic_angle", (k, theta0, min, max, tol), "Harmonic Angle")

    @staticmethod
    def harmonic_dihedral(k, n, delta, tol=0.001):
        """k (1 + cos(n phi - delta)), tabulated in cos(phi) (MxPotential.cpp:2595-2607)."""
        return Potential._make("mxg_potential_create_harmonic_dihedral", (k, int(n), delta, tol), "Harmonic Dihedral")

    @staticmethod
    def power(k=1.0, r0=1.0, alpha=1.0, min=None, max=None, tol=None):
        dmin, dmax = 0.1, 3.0
        dtol = 0.001 if alpha >= 1 else 0.01
        if r0 > 0:
            dmin = r0 if alpha <= 1 else 0.1 * r0
            dmax = 3.0 * r0
        return Potential._make("mxg_potential_create_power",
                               (k, r0, alpha, dmin if min is None else min, dmax if max is None else max,
                                dtol if tol is None else tol), "Power")

    @staticmethod
    def dpd(alpha=1.0, gamma=1.0, sigma=1.0, cutoff=1.0, shifted=False):
        # the reference stores the parameters as float (MxPotential.cpp:2738-2750)
        return Potential._make("mxg_potential_create_dpd", (alpha, gamma, sigma, cutoff, int(bool(shifted))),
                               "Dissapative Particle Dynamics")

    def __add__(self, other):
        """p1 + p2: both potentials act on the pairs they are bound to, summed
        (a table potential plus a DPD thermostat, say). No counterpart in the
        reference, which binds one potential per type pair."""
        if not isinstance(other, Potential):
            return NotImplemented
        return PotentialSum(self, other)

    def refit(self, params):
        """Frozen-node re-fit at new construction parameters (same nodes and
        interval count), so the coefficients are linear in the sampled potential."""
        q = np.ascontiguousarray(params, dtype=np.float64)
        check(lib().mxg_potential_refit(self._h, ptr(q, ctypes.c_double), len(q)), "potential_refit")

    def param_table(self, k):
        """The table of dV/dtheta_k on this table's nodes (see mxg_potential_param_table)."""
        h = ctypes.c_void_p()
        check(lib().mxg_potential_param_table(self._h, int(k), ctypes.byref(h)), "potential_param_table")
        return Potential(h.value, self.name + f" d/dparam{k}")

    def _info(self):
        kind, flags, n = ctypes.c_int(), ctypes.c_uint(), ctypes.c_int()
        a4 = (ctypes.c_float * 4)()
        a, b, r0 = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
        check(lib().mxg_potential_info(self._h, ctypes.byref(kind), ctypes.byref(flags), ctypes.byref(n), a4,
                                       ctypes.byref(a), ctypes.byref(b), ctypes.byref(r0)), "potential_info")
        return dict(kind=kind.value, flags=flags.value, n=n.value, alpha=np.array(a4, dtype=np.float32),
                    a=a.value, b=b.value, r0_plusone=r0.value)

    @property
    def min(self):
        return self._info()["a"]

    @property
    def max(self):
        return self._info()["b"]

    cutoff = max

    @property
    def domain(self):
        i = self._info()
        return (i["a"], i["b"])

    @property
    def intervals(self):
        return self._info()["n"]

    @property
    def flags(self):
        return self._info()["flags"]

    @property
    def kind(self):
        return self._info()["kind"]

    @property
    def coefficients(self):
        n = self.intervals
        out = np.zeros((n + 1) * 8, dtype=np.float32)
        check(lib().mxg_potential_coeffs(self._h, ptr(out, ctypes.c_float), out.size), "potential_coeffs")
        return out

    def __call__(self, r, r0=None):
        """(energy, force) at distance r; like potential_call (MxPotential.cpp:2375-2414)."""
        info = self._info()
        if (info["flags"] & ((1 << 11) | (1 << 12))) and (r0 is None or r0 < 0):
            r0 = 1.0
        r0 = 0.0 if r0 is None else r0
        e, f = ctypes.c_float(), ctypes.c_float()
        lib().mxg_potential_eval(self._h, r0 / 2, r0 / 2, float(np.float32(r) * np.float32(r)), ctypes.byref(e),
                                 ctypes.byref(f))
        return (e.value, float(np.float32(f.value) * np.float32(r)))


class _ConstantForce:
    def __init__(self, value, period=None):
        self.value = np.asarray(value, dtype=np.float32).reshape(3)


class _SingleBodyForce:
    """The forces module's other one-body forces (MxForce.cpp:213-259); kind and
    params as mxg_engine_add_singlebody_force_kind takes them."""

    def __init__(self, kind, params):
        self.kind = kind
        self.params = np.asarray(list(params) + [0.0] * (4 - len(params)), dtype=np.float32)


def _berenderson_tstat(tau):
    """Berendsen thermostat force (1/tau)(T0/KE_type - 1) v with T0 the type's target_temperature."""
    return _SingleBodyForce(2, [tau])


def _random(std, mean, durration=0.01):
    """A persistent random force in a random direction, redrawn every durration.
    As in the reference, the module passes (std, mean) into parameters declared
    (mean, std) (MxForce.cpp:18,226-233), so the magnitude is drawn from a normal
    distribution with mean `std` and standard deviation `mean`."""
    return _SingleBodyForce(3, [std, mean, durration])


def _friction(coef, std=0.0, mean=0.0, durration=0.01):
    """-coef |v|^2 v plus a persistent random force as for random(), with the
    reference's same (std, mean) exchange (MxForce.cpp:19,239-247)."""
    return _SingleBodyForce(4, [coef, std, mean, durration])


class forces:  # noqa: N801 - namespace mirroring m.forces
    ConstantForce = _ConstantForce
    berenderson_tstat = staticmethod(_berenderson_tstat)
    random = staticmethod(_random)
    friction = staticmethod(_friction)


class Bond:
    """A pairwise bond with a table potential and dissociation threshold
    (bond.cpp:535-560; break test eff >= dissociation_energy, bond.cpp:230)."""

    def __init__(self, potential, i, j, dissociation_energy=np.finfo(np.float64).max):
        u = _require()
        self.id = u._add_bonds(potential, [_pid(i)], [_pid(j)], dissociation_energy)[0]
        self.potential = potential

    @property
    def active(self):
        return bool(universe.bond_flags()[self.id] & 1)

    @classmethod
    def _handle(cls, bond_id, potential):
        b = cls.__new__(cls)
        b.id = bond_id
        b.potential = potential
        return b


def _ids_of(particles):
    """Particle ids of a particle, a list/tuple of particles or ids, or an id array."""
    if isinstance(particles, Particle):
        return np.array([particles.id], dtype=np.int32)
    if isinstance(particles, np.ndarray):
        return np.ascontiguousarray(particles, dtype=np.int32).ravel()
    if isinstance(particles, (list, tuple)):
        return np.array([_pid(p) for p in particles], dtype=np.int32)
    raise TypeError("argument 1 is not a particle list")


class Angle:
    """An angle p1-p2-p3 with its vertex at p2 and a potential in cos(theta)
    (angle.cpp:659-707); evaluated every force pass after the bonds
    (angle_eval, angle.cpp:92-352)."""

    def __init__(self, potential, p1, p2, p3):
        if not isinstance(potential, Potential):
            raise TypeError("potential is not a instance of Potential")
        u = _require()
        self.i, self.j, self.k = _pid(p1), _pid(p2), _pid(p3)
        self.id = u._add_angles(potential, [self.i], [self.j], [self.k])[0]
        self.potential = potential


class Dihedral:
    """A dihedral p1-p2-p3-p4 with a potential in cos(phi) between the planes
    (p1, p2, p3) and (p2, p3, p4), evaluated every force pass after the angles
    (dihedral_eval, dihedral.cpp:81-392). The reference reaches dihedrals through
    engine_dihedral_addpot / engine_dihedral_add (engine_bonded.cpp:1049-1080,
    1967-1991) and its file readers; it has no Python constructor for them."""

    def __init__(self, potential, p1, p2, p3, p4):
        if not isinstance(potential, Potential):
            raise TypeError("potential is not a instance of Potential")
        u = _require()
        self.i, self.j, self.k, self.l = _pid(p1), _pid(p2), _pid(p3), _pid(p4)
        self.id = u._add_dihedrals(potential, [self.i], [self.j], [self.k], [self.l])[0]
        self.potential = potential


class Cuboid:
    """A static box that particles of a bound type are pushed from (the reference's Cuboid,
    MxCuboid.cpp:40-76): centre pos (default the box centre, engine_center), size and the
    orientation angles about x, y and z. Bind a potential to it with
    bind(potential, Cuboid, ParticleType)."""

    def __init__(self, pos=None, size=(1.0, 1.0, 1.0), orientation=(0.0, 0.0, 0.0), replica=0):
        self.id = _require()._add_cuboid(pos, size, orientation, replica)

    @property
    def geometry(self):
        return universe.cuboid_info(self.id)


class BoundaryCondition:
    """One face of the box (MxBoundaryCondition, MxBoundaryConditions.hpp:25-52);
    ``bind(potential, face, Type)`` puts a wall potential between the face and
    the type's particles."""

    _NORMALS = ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1))

    def __init__(self, face):
        self.face = face
        self.name = _FACES[face]
        self.normal = np.array(self._NORMALS[face], dtype=np.float32)


class BoundaryConditions:
    """The six faces (MxBoundaryConditions); ``bind(potential, universe.boundary_conditions,
    Type)`` binds the wall potential on every face (MxBoundaryConditions.cpp:828-837)."""

    def __init__(self):
        for f, name in enumerate(_FACES):
            setattr(self, name, BoundaryCondition(f))


def _pid(p):
    return p.id if isinstance(p, Particle) else int(p)


class _SpeciesView:
    """A particle's species values by name (``p.species.S1``, ``p.species.S1 = 0.5``)."""

    def __init__(self, pid, tid):
        object.__setattr__(self, "_pid", pid)
        object.__setattr__(self, "_tid", tid)

    def _index(self, name):
        return universe._species_index(self._tid, name)[1]

    def __getattr__(self, name):
        if name.startswith("_"):
            raise AttributeError(name)
        k = self._index(name)
        if universe._started and not universe._dirty:
            return float(universe.species_values()[self._pid, k])
        return float(universe._spec[self._pid, k])

    def __setattr__(self, name, value):
        k = self._index(name)
        universe._sync_state()
        universe._spec[self._pid, k] = float(value)
        if universe._started and not universe._dirty:
            universe.set_species_values(universe._spec)


class _SpeciesAttr:
    """``Type.species`` is the type's species list; ``particle.species`` its values."""

    def __init__(self, names):
        self.names = list(names)

    def __get__(self, obj, cls=None):
        if obj is None:
            return self.names
        return _SpeciesView(obj.id, type(obj).id)


class _ParticleMeta(type):
    def __init__(cls, name, bases, ns):
        super().__init__(name, bases, ns)
        if bases and any(isinstance(b, _ParticleMeta) for b in bases):
            u = _require()
            cls.id = u._add_type(cls)
            if isinstance(ns.get("species"), (list, tuple)):
                cls.species = _SpeciesAttr(ns["species"])

    def factory(cls, positions=None, velocities=None, nr_parts=None, replica=0):
        """Bulk creation of particles of this type from arrays (N x 3)."""
        u = _require()
        x = np.asarray(positions, dtype=np.float64).reshape(-1, 3)
        v = np.zeros_like(x, dtype=np.float32) if velocities is None else np.asarray(velocities).reshape(-1, 3)
        ids = u._add_particles(x, v, np.full(len(x), cls.id, dtype=np.int32), replica)
        return ids

    def items(cls):
        """This type's particles, in id order, as a ParticleList (ParticleType.items)."""
        return ParticleList(np.flatnonzero(_require()._t == cls.id).astype(np.int32))


class ParticleList:
    """A list of particle ids with the reference's group metrics (MxParticleList,
    src/mdcore/src/MxParticleList.cpp:193-199), computed on the device over the
    current state: centre of mass, centroid, radius of gyration and moment of
    inertia with the formulas of src/mdcore/src/metrics.cpp:330-466 (the radius of
    gyration is the square root of the summed distances to the centroid, and the
    inertia's off-diagonal terms are + sum m dx dy, as there). Behaves as an int32
    array of the ids."""

    def __init__(self, ids):
        self.ids = np.ascontiguousarray(np.asarray(ids, dtype=np.int32).reshape(-1))

    def __len__(self):
        return len(self.ids)

    def __iter__(self):
        return iter(self.ids.tolist())

    def __getitem__(self, k):
        return self.ids[k]

    def __array__(self, dtype=None, copy=None):
        return self.ids if dtype is None else self.ids.astype(dtype)

    def __repr__(self):
        return f"ParticleList({self.ids.tolist()!r})"

    def _metrics(self):
        if len(self.ids) == 0:
            raise ValueError("empty particle list")
        u = _require()
        u._ensure()
        out = np.zeros(17)
        check(lib().mxg_engine_group_metrics(u._e, len(self.ids), ptr(self.ids, ctypes.c_int),
                                             out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), "group_metrics")
        return out

    def center_of_mass(self):
        return self._metrics()[1:4]

    def centroid(self):
        return self._metrics()[4:7]

    def radius_of_gyration(self):
        return float(self._metrics()[7])

    def moment_of_inertia(self):
        return self._metrics()[8:17].reshape(3, 3)

    inertia = moment_of_inertia


class Particle(metaclass=_ParticleMeta):
    """Base particle type; subclasses define a type (mass, radius, dynamics)."""

    mass = 1.0
    radius = 1.0
    dynamics = Newtonian
    frozen = 0

    def __init__(self, position=None, velocity=None):
        u = _require()
        if position is None:
            position = np.random.uniform(0, 1, 3) * np.asarray(u.dim)
        velocity = np.zeros(3) if velocity is None else velocity
        self.id = u._add_particles(np.asarray(position, dtype=np.float64).reshape(1, 3),
                                   np.asarray(velocity, dtype=np.float32).reshape(1, 3),
                                   np.array([type(self).id], dtype=np.int32))[0]

    @property
    def position(self):
        return universe.positions[self.id]

    @property
    def velocity(self):
        return universe.velocities[self.id]

    @property
    def force(self):
        return universe.forces[self.id]


class _Universe:
    """The simulation (engine + space); mirrors MxUniverse."""

    def __init__(self):
        self._e = None

    # ---- configuration ----
    def _init(self, dim, cells, cutoff, dt, bc, max_distance, origin, rng, max_types, stream=None, pair_pruning=0,
              integrator=FORWARD_EULER):
        self.stream = stream
        self.integrator = int(integrator)
        self.pair_pruning = pair_pruning
        self.dim = [float(d) for d in dim]
        self.origin = [float(o) for o in origin]
        self.cells = [int(c) for c in cells]
        self.cutoff = float(cutoff)
        self.dt = float(dt)
        self.bc = bc
        self.max_distance = max_distance
        self.rng = rng
        self.max_types = max_types
        self.time = 0
        self._types = []        # (mass, radius, dynamics, flags)
        self._pots = []         # (potential, ti, tj, replica)
        self._replicas = []     # extra boxes: (origin, dim, cells, bc)
        self._forces = []       # (type, force object), one per type
        self._targets = {}      # type -> target temperature
        self._bonds = []        # (potential, i[], j[], dissociation)
        self._angles = []       # (potential, i[], j[], k[])
        self._dihedrals = []    # (potential, i[], j[], k[], l[])
        self._exclusions = []   # (i[], j[])
        self._bpots = []        # wall potentials: (potential, face or -1, type)
        self._cuboids = []      # (replica, pos or None, size, angles)
        self._cuboid_pots = []  # (potential, type)
        self._species = {}      # type -> (species names, flags)
        self._spec_width = 0
        self._spec = np.zeros((0, 0), dtype=np.float32)  # species values by particle id
        self._fluxes = []       # (kind, type a, type b, species a, species b, k, decay, target)
        self._x = np.zeros((0, 3))
        self._v = np.zeros((0, 3), dtype=np.float32)
        self._t = np.zeros(0, dtype=np.int32)
        self._r = np.zeros(0, dtype=np.int32)
        self._c = np.zeros(0, dtype=np.int32)  # given cell of a particle added cell-relative, else -1
        self._xr = np.zeros((0, 3), dtype=np.float32)  # its cell-relative position
        self.occupancy_hint = 0  # particle count the force pass's work-item split is decided on (0: own)
        self._started = False
        self._dirty = False
        self._new_engine()

    def _new_engine(self):
        if self._e is not None:
            lib().mxg_engine_finalize(self._e)
            self._e = None
        kind, vel, restore = parse_bc(self.bc)
        h = ctypes.c_void_p()
        check(lib().mxg_engine_init(ptr(f64(self.origin), ctypes.c_double), ptr(f64(self.dim), ctypes.c_double),
                                    ptr(i32(self.cells), ctypes.c_int), self.cutoff, ptr(i32(kind), ctypes.c_int),
                                    ptr(f32(vel), ctypes.c_float), ptr(f32(restore), ctypes.c_float),
                                    self.max_types, 0, ctypes.byref(h)), "engine_init")
        self._e = h
        _LIVE.add(self)
        frac = -1.0
        if self.max_distance is not None and self.max_distance >= 0:
            hh = self.space_info()[1]
            frac = self.max_distance / hh[0]
        check(lib().mxg_engine_set_dt(self._e, self.dt, frac), "set_dt")
        check(lib().mxg_engine_set_rng_mode(self._e, 1 if self.rng == "philox" else 0), "set_rng_mode")
        check(lib().mxg_engine_set_pair_pruning(self._e, int(self.pair_pruning)), "set_pair_pruning")
        check(lib().mxg_engine_set_integrator(self._e, int(self.integrator)), "set_integrator")
        for (o, d, c, b) in self._replicas:
            kind, vel, restore = parse_bc(b)
            check(lib().mxg_engine_add_replica(self._e, ptr(f64(o), ctypes.c_double), ptr(f64(d), ctypes.c_double),
                                               ptr(i32(c), ctypes.c_int), ptr(i32(kind), ctypes.c_int),
                                               ptr(f32(vel), ctypes.c_float), ptr(f32(restore), ctypes.c_float)),
                  "add_replica")
        for (m, r, d, fl) in self._types:
            check(lib().mxg_engine_addtype(self._e, m, r, d, fl), "addtype")
        for (p, a, b, rep, which) in self._pots:
            if which == 0:
                check(lib().mxg_engine_addpot_replica(self._e, rep, p._h, a, b), "addpot")
            else:
                check(lib().mxg_engine_addpot_second(self._e, rep, p._h, a, b), "addpot_second")
        for (t, f) in self._forces:
            if isinstance(f, _SingleBodyForce):
                check(lib().mxg_engine_add_singlebody_force_kind(self._e, t, f.kind, ptr(f.params, ctypes.c_float)),
                      "add_singlebody_force")
            else:
                v = f.value
                check(lib().mxg_engine_add_singlebody_force(self._e, t, float(v[0]), float(v[1]), float(v[2])),
                      "add_singlebody_force")
        for t, temp in self._targets.items():
            check(lib().mxg_engine_set_target_temperature(self._e, t, float(temp)), "set_target_temperature")
        for (p, ii, jj, d) in self._bonds:
            check(lib().mxg_engine_addbonds(self._e, len(ii), ptr(ii, ctypes.c_int), ptr(jj, ctypes.c_int), p._h, d,
                                            None), "addbonds")
        for (p, ii, jj, kk) in self._angles:
            check(lib().mxg_engine_addangles(self._e, len(ii), ptr(ii, ctypes.c_int), ptr(jj, ctypes.c_int),
                                             ptr(kk, ctypes.c_int), p._h, None), "addangles")
        for t, (names, flags) in self._species.items():
            fl = np.asarray(flags, dtype=np.uint32)
            check(lib().mxg_engine_set_type_species(self._e, t, len(names), fl.ctypes.data_as(ctypes.c_void_p)),
                  "set_type_species")
        for f in self._fluxes:
            check(lib().mxg_engine_add_flux(self._e, *f), "add_flux")
        for (p, face, t) in self._bpots:
            check(lib().mxg_engine_set_boundary_potential(self._e, face, t, p._h), "set_boundary_potential")
        for (rep, pos, size, ang) in self._cuboids:
            check(lib().mxg_engine_add_cuboid(self._e, rep, None if pos is None else ptr(f32(pos), ctypes.c_float),
                                              ptr(f32(size), ctypes.c_float), ptr(f32(ang), ctypes.c_float), None),
                  "add_cuboid")
        for (p, t) in self._cuboid_pots:
            check(lib().mxg_engine_set_cuboid_potential(self._e, t, p._h), "set_cuboid_potential")
        for (ii, jj) in self._exclusions:
            check(lib().mxg_engine_add_exclusions(self._e, len(ii), ptr(ii, ctypes.c_int), ptr(jj, ctypes.c_int)),
                  "add_exclusions")
        for (p, ii, jj, kk, ll) in self._dihedrals:
            check(lib().mxg_engine_adddihedrals(self._e, len(ii), ptr(ii, ctypes.c_int), ptr(jj, ctypes.c_int),
                                                ptr(kk, ctypes.c_int), ptr(ll, ctypes.c_int), p._h, None),
                  "adddihedrals")
        self._started = False

    def _add_type(self, cls):
        fl = int(getattr(cls, "frozen", 0))
        rec = (float(cls.mass), float(cls.radius), int(cls.dynamics), fl)
        tid = check(lib().mxg_engine_addtype(self._e, *rec), "addtype") if not self._started else None
        self._types.append(rec)
        if tid is None:
            self._dirty = True
            tid = len(self._types) - 1
        names = getattr(cls, "species", None)
        if isinstance(names, _SpeciesAttr):
            names = names.names
        if names:
            # species list ("$" marks a constant species, SPECIES_KONSTANT)
            names = [str(s) for s in names]
            self._species[tid] = ([s.lstrip("$") for s in names], [4 if s.startswith("$") else 0 for s in names])
            self._spec_width = max(self._spec_width, len(names))
            if self._spec.shape[1] < self._spec_width:
                self._spec = np.pad(self._spec, ((0, 0), (0, self._spec_width - self._spec.shape[1])))
            self._dirty = True
        if getattr(cls, "target_temperature", None) is not None:
            self._targets[tid] = float(cls.target_temperature)
            if self._started:
                self._dirty = True
            else:
                check(lib().mxg_engine_set_target_temperature(self._e, tid, self._targets[tid]), "target_temperature")
        return tid

    def _add_particles(self, x, v, t, replica=0):
        first = len(self._t)
        self._sync_state()
        self._spec = np.concatenate([self._spec, np.zeros((len(t), self._spec.shape[1]), dtype=np.float32)])
        self._x = np.concatenate([self._x, np.asarray(x, dtype=np.float64)])
        self._v = np.concatenate([self._v, np.asarray(v, dtype=np.float32)])
        self._t = np.concatenate([self._t, np.asarray(t, dtype=np.int32)])
        self._r = np.concatenate([self._r, np.full(len(t), int(replica), dtype=np.int32)])
        self._c = np.concatenate([self._c, np.full(len(t), -1, dtype=np.int32)])
        self._xr = np.concatenate([self._xr, np.zeros((len(t), 3), dtype=np.float32)])
        self._dirty = True
        return list(range(first, first + len(t)))

    def _add_particles_cellrel(self, cell, xrel, v, t, replica=0):
        """Adds particles by cell (the engine's cell index in the replica) and FP32 cell-relative
        position, kept exactly as given (mxg_engine_addparts_cellrel): a state handed over from
        another engine over the same space continues bit for bit."""
        cell = np.asarray(cell, dtype=np.int32)
        xrel = np.asarray(xrel, dtype=np.float32).reshape(-1, 3)
        cdim, h = self.cell_grid()
        loc = np.stack([cell // (cdim[1] * cdim[2]), (cell // cdim[2]) % cdim[1], cell % cdim[2]], axis=1)
        x = np.asarray(self.origin) + loc * h + xrel.astype(np.float64)  # the global positions they stand for
        k0 = len(self._t)
        first = self._add_particles(x, v, t, replica)
        self._c[k0:] = cell
        self._xr[k0:] = xrel
        return first

    def cell_grid(self):
        """(cells per axis, cell edge) of the engine's grid (space_init's cdim and h)."""
        cdim = (ctypes.c_int * 3)()
        h = (ctypes.c_double * 3)()
        nc = ctypes.c_int()
        per = ctypes.c_uint()
        check(lib().mxg_engine_space_info(self._e, cdim, h, ctypes.byref(nc), ctypes.byref(per)), "space_info")
        return np.array(cdim[:], dtype=np.int64), np.array(h[:])

    def add_replica(self, dim, cells, bc=None, origin=(0.0, 0.0, 0.0)):
        """Adds an independent simulation box that steps together with the others
        (batched ensembles); returns its replica index. Types, cutoff and dt are shared."""
        self._sync_state()
        self._replicas.append((list(origin), list(dim), list(cells), bc))
        self._dirty = True
        return len(self._replicas)

    def _add_bonds(self, pot, i, j, d):
        ii, jj = i32(i), i32(j)
        first = sum(len(b[1]) for b in self._bonds)
        self._bonds.append((pot, ii, jj, float(d)))
        self._sync_state()
        self._dirty = True
        return list(range(first, first + len(ii)))

    # ---- species (chemical cargo) and fluxes ----
    def _species_index(self, cls, name):
        t = cls.id if isinstance(cls, type) else int(cls)
        if t not in self._species:
            raise ValueError(f"particle type {getattr(cls, '__name__', t)} does not have any defined species")
        names = self._species[t][0]
        if name not in names:
            raise ValueError(f"particle type {getattr(cls, '__name__', t)} does not have species {name}")
        return t, names.index(name)

    def _add_flux(self, kind, a, b, name, k, decay, target):
        ta, ia = self._species_index(a, name)
        tb, ib = self._species_index(b, name)
        key = (min(ta, tb), max(ta, tb))
        if sum(1 for f in self._fluxes if (min(f[1], f[2]), max(f[1], f[2])) == key) + 1 >= 8:
            raise ValueError("at most 7 fluxes per pair of types")  # MxFluxes_AddFlux's limit
        self._sync_state()
        self._fluxes.append((int(kind), ta, tb, ia, ib, float(k), float(decay), float(target)))
        self._dirty = True

    def species_values(self):
        """Species values by particle id (N x the widest type's species count)."""
        self._ensure()
        if not self._spec_width:
            return np.zeros((len(self._t), 0), dtype=np.float32)
        out = np.zeros((len(self._t), self._spec.shape[1]), dtype=np.float32)
        check(lib().mxg_engine_get_species(self._e, len(self._t), out.shape[1], ptr(out, ctypes.c_float)),
              "get_species")
        return out

    def set_species_values(self, values):
        """Replaces the species values (N x width, by particle id)."""
        vals = np.ascontiguousarray(values, dtype=np.float32)
        self._spec = vals.copy()
        if self._started and not self._dirty:
            check(lib().mxg_engine_set_species(self._e, vals.shape[0], vals.shape[1], ptr(vals, ctypes.c_float)),
                  "set_species")

    @property
    def boundary_conditions(self):
        """The box faces, for binding wall potentials (Universe.boundary_conditions)."""
        return BoundaryConditions()

    def _add_angles(self, pot, i, j, k):
        ii, jj, kk = i32(i), i32(j), i32(k)
        first = sum(len(a[1]) for a in self._angles)
        self._angles.append((pot, ii, jj, kk))
        self._sync_state()
        self._dirty = True
        return list(range(first, first + len(ii)))

    def add_exclusions(self, i, j):
        """Excludes the pairs (i[q], j[q]) from the pair potential: each force pass takes the
        pair's table potential back (engine_exclusion_add and exclusion_eval; the reference
        reaches them from C and its file readers only)."""
        ii = i32([_pid(p) for p in np.atleast_1d(i)])
        jj = i32([_pid(p) for p in np.atleast_1d(j)])
        self._sync_state()
        self._exclusions.append((ii, jj))
        self._dirty = True

    def _add_dihedrals(self, pot, i, j, k, l):
        ii, jj, kk, ll = i32(i), i32(j), i32(k), i32(l)
        first = sum(len(d[1]) for d in self._dihedrals)
        self._dihedrals.append((pot, ii, jj, kk, ll))
        self._sync_state()
        self._dirty = True
        return list(range(first, first + len(ii)))

    def bind_pairwise(self, potential, particles, cutoff, pairs=None, half_life=None, bond_energy=None, flags=0):
        """Bonds every pair of the listed particles within cutoff of each other
        (Universe.bind_pairwise, MxUniverse.cpp:669-733; MxBond_PairwiseNew,
        bond.cpp:944-989). The pair search runs on the device over the current
        state (global FP32 positions, no periodic image, pairs (a, b) with b
        before a in the list, ordered by a then b); pairs: optional list of
        (type, type) tuples that restricts the bonded type pairs. bond_energy is
        the bonds' dissociation energy (default: never break). Returns the new
        Bond handles."""
        if not isinstance(potential, Potential):
            raise TypeError("argument 0 is not a potential")
        ids = _ids_of(particles)
        self._ensure()
        nt, mask = 0, None
        if pairs is not None:
            nt = len(self._types)
            mask = np.zeros((nt, nt), dtype=np.uint8)
            for (ta, tb) in pairs:
                a = ta.id if isinstance(ta, type) else int(ta)
                b = tb.id if isinstance(tb, type) else int(tb)
                mask[a, b] = mask[b, a] = 1
        mptr = None if mask is None else mask.ctypes.data_as(ctypes.c_void_p)
        count = ctypes.c_int()
        check(lib().mxg_engine_pairs_within(self._e, len(ids), ptr(ids, ctypes.c_int), float(cutoff), mptr, nt,
                                            None, None, 0, ctypes.byref(count)), "pairs_within")
        bi = np.zeros(count.value, dtype=np.int32)
        bj = np.zeros(count.value, dtype=np.int32)
        if count.value:
            check(lib().mxg_engine_pairs_within(self._e, len(ids), ptr(ids, ctypes.c_int), float(cutoff), mptr, nt,
                                                ptr(bi, ctypes.c_int), ptr(bj, ctypes.c_int), count.value,
                                                ctypes.byref(count)), "pairs_within")
        d = np.finfo(np.float64).max if bond_energy is None else float(bond_energy)
        new = self._add_bonds(potential, bi, bj, d) if count.value else []
        return [Bond._handle(k, potential) for k in new]

    def _add_cuboid(self, pos, size, orientation, replica=0):
        self._sync_state()
        self._cuboids.append((int(replica), None if pos is None else [float(q) for q in pos],
                              [float(q) for q in size], [float(q) for q in orientation]))
        self._dirty = True
        return len(self._cuboids) - 1

    def cuboid_info(self, k):
        """(centre, size, orientation quaternion (x, y, z, w), box min, box max) of cuboid k."""
        self._ensure()
        out = np.zeros(16, dtype=np.float32)
        check(lib().mxg_engine_cuboid_info(self._e, int(k), ptr(out, ctypes.c_float)), "cuboid_info")
        return out[0:3], out[3:6], out[6:10], out[10:13], out[13:16]

    def bind(self, obj, a, b=None, replica=0):
        """Binds a potential to a pair of types, to a type and a wall (a
        BoundaryCondition face or all of BoundaryConditions), to a type and the cuboids
        (bind(pot, Cuboid, type)), or a force to a type (MxBind.cpp:18-100)."""
        if isinstance(obj, Potential) and (a is Cuboid or b is Cuboid):
            t = b if a is Cuboid else a
            self._sync_state()
            self._cuboid_pots = [(p, q) for (p, q) in self._cuboid_pots if q != t.id]  # one per type
            self._cuboid_pots.append((obj, t.id if isinstance(t, type) else int(t)))
            self._dirty = True
            return
        walls = (BoundaryCondition, BoundaryConditions)
        if isinstance(obj, Potential) and (isinstance(a, walls) or isinstance(b, walls)):
            bc, t = (a, b) if isinstance(a, walls) else (b, a)
            ti = t.id if isinstance(t, type) else int(t)
            self._sync_state()
            self._bpots.append((obj, bc.face if isinstance(bc, BoundaryCondition) else -1, ti))
            self._dirty = True
            return
        ta = a.id if isinstance(a, type) else int(a)
        if isinstance(obj, (Potential, PotentialSum)):
            tb = ta if b is None else (b.id if isinstance(b, type) else int(b))
            self._sync_state()
            terms = obj.terms if isinstance(obj, PotentialSum) else (obj,)
            for which, p in enumerate(terms):
                self._pots.append((p, ta, tb, int(replica), which))
            self._dirty = True
        elif isinstance(obj, (_ConstantForce, _SingleBodyForce)):
            self._sync_state()
            self._forces = [(t, f) for (t, f) in self._forces if t != ta]  # one single-body force per type
            self._forces.append((ta, obj))
            self._dirty = True
        else:
            raise TypeError("bind expects a Potential or a force")

    def potential_index(self, a, b, replica=0, which=0):
        """The engine's index of the potential bound to types (a, b)."""
        self._ensure()
        ta = a.id if isinstance(a, type) else int(a)
        tb = b.id if isinstance(b, type) else int(b)
        idx = ctypes.c_int()
        check(lib().mxg_engine_pot_index(self._e, int(replica), ta, tb, int(which), ctypes.byref(idx)), "pot_index")
        return idx.value

    def bond_potential_indices(self, pot):
        """The engine's indices of the copies of pot that bonds use (one per group of bonds
        created together)."""
        self._ensure()
        out, first = [], 0
        for (p, ii, jj, d) in self._bonds:
            if p is pot and len(ii):
                idx = ctypes.c_int()
                check(lib().mxg_engine_bond_pot_index(self._e, first, ctypes.byref(idx)), "bond_pot_index")
                out.append(idx.value)
            first += len(ii)
        return out

    def set_bond_flags(self, flags):
        """Replaces the bonds' active flags (one per bond, in creation order)."""
        self._ensure()
        f = np.ascontiguousarray(flags, dtype=np.uint32)
        check(lib().mxg_engine_set_bond_flags(self._e, ptr(f, ctypes.c_uint), len(f)), "set_bond_flags")

    def set_potential_params(self, pot, params):
        """New construction parameters for a bound potential: the host object is
        re-fitted on its frozen nodes and every engine copy of it (type pairs and
        bonds) is updated in place."""
        q = np.ascontiguousarray(params, dtype=np.float64)
        pot.refit(q)
        if self._e is None or self._dirty or not self._started:
            self._dirty = True
            return
        idxs = [self.potential_index(a, b, rep, which) for (p, a, b, rep, which) in self._pots if p is pot]
        for idx in idxs + self.bond_potential_indices(pot):
            check(lib().mxg_engine_set_pot_params(self._e, idx, ptr(q, ctypes.c_double), len(q)), "set_pot_params")

    # ---- engine lifecycle ----
    def _sync_state(self):
        """Pulls the device state back into the host arrays before a rebuild."""
        if self._started:
            n = len(self._t)
            x = np.zeros((n, 3))
            v = np.zeros((n, 3), dtype=np.float32)
            check(lib().mxg_engine_unload(self._e, n, ptr(x, ctypes.c_double), ptr(v, ctypes.c_float), None, None,
                                          None), "unload")
            self._x, self._v = x, v
            self._c[:] = -1  # the pulled global positions now stand for every particle
            if self._spec_width and self._spec.shape[1]:
                sp = np.zeros((n, self._spec.shape[1]), dtype=np.float32)
                check(lib().mxg_engine_get_species(self._e, n, sp.shape[1], ptr(sp, ctypes.c_float)), "get_species")
                self._spec = sp

    def _ensure(self):
        if self._started and not self._dirty:
            return
        if self._started or self._dirty:
            self._new_engine()
        n = len(self._t)
        # particles go in id order; consecutive runs of one replica (and of one way of placing them)
        # are added together
        k = 0
        while k < n:
            rep = int(self._r[k])
            given = self._c[k] >= 0
            e = k
            while e < n and self._r[e] == rep and (self._c[e] >= 0) == given:
                e += 1
            if given:
                check(lib().mxg_engine_addparts_cellrel(self._e, rep, e - k, ptr(i32(self._c[k:e]), ctypes.c_int),
                                                        ptr(f32(self._xr[k:e]), ctypes.c_float),
                                                        ptr(f32(self._v[k:e]), ctypes.c_float),
                                                        ptr(i32(self._t[k:e]), ctypes.c_int), None), "addparts")
            else:
                check(lib().mxg_engine_addparts_replica(self._e, rep, e - k, ptr(f64(self._x[k:e]), ctypes.c_double),
                                                        ptr(f32(self._v[k:e]), ctypes.c_float),
                                                        ptr(i32(self._t[k:e]), ctypes.c_int), None), "addparts")
            k = e
        if self.occupancy_hint:
            check(lib().mxg_engine_set_occupancy_hint(self._e, int(self.occupancy_hint)), "occupancy_hint")
        if self._spec_width:
            sp = np.ascontiguousarray(self._spec, dtype=np.float32)
            check(lib().mxg_engine_set_species(self._e, n, sp.shape[1], ptr(sp, ctypes.c_float)), "set_species")
        check(lib().mxg_engine_start(self._e, ctypes.c_void_p(self.stream) if self.stream else None),
              "engine_start")
        self._started = True
        self._dirty = False

    @property
    def handle(self):
        self._ensure()
        return self._e

    def step(self, until=0, dt=0):
        """One engine step (MxUniverse_Step ignores until and dt, MxUniverse.cpp:549-566)."""
        self.steps(1)

    def steps(self, n):
        self._ensure()
        check(lib().mxg_engine_step(self._e, int(n)), "engine_step")
        self.time += int(n)
        check(lib().mxg_engine_status(self._e), "engine_step")

    def number_density(self):
        """(number density by particle id, computed volume) for the current positions: the
        reference's per-particle f[3] (W(0, cutoff) plus W(r^2, cutoff) over the pairs the
        pair loops reach) and the sum of its inverses (engine_advance.cpp:184-185)."""
        self._ensure()
        n = len(self._t)
        out = np.zeros(n, dtype=np.float32)
        vol = ctypes.c_double()
        check(lib().mxg_engine_number_density(self._e, n, ptr(out, ctypes.c_float), ctypes.byref(vol)),
              "number_density")
        return out, vol.value

    def load(self, x, v=None):
        """Replaces every particle's position (global coordinates, by id) and, when given, its
        velocity (engine_load, engine.cpp:472-618): the particles are re-placed in their
        cells on the device as engine_addpart places them."""
        self._ensure()
        xx = f64(np.asarray(x).reshape(-1, 3))
        vv = None if v is None else f32(np.asarray(v).reshape(-1, 3))
        check(lib().mxg_engine_load(self._e, len(xx), ptr(xx, ctypes.c_double),
                                    None if vv is None else ptr(vv, ctypes.c_float)), "engine_load")

    def device_state(self):
        """Zero-copy torch views of the device-resident state in slot order (cells in order,
        ascending id inside a cell): "pos" (N, 4) float32 cell-relative x, y, z and the type id's
        bits in w; "vel" (N, 4) v and the particle id's bits in w; "force" (N, 4); "cell" (N,)
        int32. Read the w columns with .view(torch.int32). The views follow the engine's double
        buffers, so they are valid until the next step or force pass."""
        import torch
        self._ensure()
        p, v, f, c = (ctypes.c_void_p() for _ in range(4))
        check(lib().mxg_engine_device_state(self._e, ctypes.byref(p), ctypes.byref(v), ctypes.byref(f),
                                            ctypes.byref(c)), "device_state")
        n = len(self._t)

        class _View:
            def __init__(self, ptr, shape, typestr):
                self.__cuda_array_interface__ = {"shape": shape, "typestr": typestr, "data": (ptr, False),
                                                 "version": 3, "strides": None}

        out = {}
        for name, ptr_, shape, ts in (("pos", p, (n, 4), "<f4"), ("vel", v, (n, 4), "<f4"),
                                      ("force", f, (n, 4), "<f4"), ("cell", c, (n,), "<i4")):
            out[name] = torch.as_tensor(_View(ptr_.value or 0, shape, ts), device="cuda")
        return out

    def checkpoint(self, path=None):
        """The exact engine state: positions and velocities in the engine's cell frame, cell
        lists, id map, step counter (which keys the random streams), bond flags, species values
        and rates and the persistent random single-body forces. Restoring it into a universe
        built the same way resumes the trajectory bit for bit. Returns a dict of arrays and
        writes it to `path` (.npz) when given. The reference has no checkpoint."""
        import torch
        self._ensure()
        b = ctypes.c_size_t()
        check(lib().mxg_engine_snapshot_bytes(self._e, ctypes.byref(b)), "snapshot_bytes")
        buf = torch.empty(b.value, dtype=torch.uint8, device="cuda")
        check(lib().mxg_engine_snapshot(self._e, ctypes.c_void_p(buf.data_ptr()), 1), "snapshot")
        check(lib().mxg_engine_status(self._e), "snapshot")  # the engine stream is done with it
        data = {"snapshot": buf.cpu().numpy(), "species": self.species_values(), "time": np.int64(self.time),
                "nparts": np.int64(len(self._t))}
        if path is not None:
            np.savez(path, **data)
        return data

    def restore(self, data):
        """Makes a checkpoint (the dict or an .npz path) the current state; the universe must
        have been built the same way (types, particles, potentials, bonds, box)."""
        import torch
        if not isinstance(data, dict):
            with np.load(data) as z:
                data = {k: z[k] for k in z.files}
        self._ensure()
        if int(data["nparts"]) != len(self._t):
            raise ValueError("the checkpoint holds a different number of particles")
        b = ctypes.c_size_t()
        check(lib().mxg_engine_snapshot_bytes(self._e, ctypes.byref(b)), "snapshot_bytes")
        snap = np.ascontiguousarray(data["snapshot"], dtype=np.uint8)
        if snap.size != b.value:
            raise ValueError("the checkpoint was taken from a differently built universe")
        buf = torch.from_numpy(snap).to("cuda")
        torch.cuda.synchronize()
        check(lib().mxg_engine_snapshot(self._e, ctypes.c_void_p(buf.data_ptr()), 0), "restore")
        check(lib().mxg_engine_status(self._e), "restore")
        self._spec = np.ascontiguousarray(data["species"], dtype=np.float32).copy()
        self.time = int(data["time"])

    def timers(self, n=1):
        """Steps n times launching kernel by kernel and returns the milliseconds per step of each
        phase, named after the reference's engine timers (engine.h:113-135)."""
        self._ensure()
        ms = np.zeros(16)
        check(lib().mxg_engine_step_timed(self._e, int(n), ptr(ms, ctypes.c_double), len(ms)), "step_timed")
        self.time += int(n)
        check(lib().mxg_engine_status(self._e), "engine_step")
        k = max(1, int(n))
        return {"step": ms[0] / k, "prepare": ms[1] / k, "nonbond": ms[4] / k, "bonded": ms[5] / k,
                "advance": ms[11] / k, "shuffle": ms[14] / k}

    def force(self):
        self._ensure()
        check(lib().mxg_engine_force(self._e), "engine_force")
        check(lib().mxg_engine_status(self._e), "engine_force")

    def _unload(self):
        self._ensure()
        n = len(self._t)
        x = np.zeros((n, 3))
        v = np.zeros((n, 3), dtype=np.float32)
        f = np.zeros((n, 3), dtype=np.float32)
        c = np.zeros(n, dtype=np.int32)
        xr = np.zeros((n, 3), dtype=np.float32)
        check(lib().mxg_engine_unload(self._e, n, ptr(x, ctypes.c_double), ptr(v, ctypes.c_float),
                                      ptr(f, ctypes.c_float), ptr(c, ctypes.c_int), ptr(xr, ctypes.c_float)), "unload")
        return x, v, f, c, xr

    @property
    def positions(self):
        return self._unload()[0]

    @property
    def velocities(self):
        return self._unload()[1]

    @property
    def forces(self):
        return self._unload()[2]

    def state(self):
        """(positions, velocities, forces, cell, cell-relative positions) by particle id."""
        return self._unload()

    def virial(self):
        """The nonbonded pair virial (3x3, FP64) of the current positions."""
        self._ensure()
        out = np.zeros(9)
        check(lib().mxg_engine_energy(self._e, None, None, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
              "virial")
        return out.reshape(3, 3)

    def energies(self):
        self._ensure()
        ep, ek = ctypes.c_double(), ctypes.c_double()
        check(lib().mxg_engine_energy(self._e, ctypes.byref(ep), ctypes.byref(ek), None), "energy")
        return ep.value, ek.value

    @property
    def kinetic_energy(self):
        return self.energies()[1]

    @property
    def potential_energy(self):
        return self.energies()[0]

    def tasks(self):
        n = lib().mxg_engine_tasks(self._e, None, 0)
        out = np.zeros(4 * n, dtype=np.int32)
        check(lib().mxg_engine_tasks(self._e, ptr(out, ctypes.c_int), out.size), "tasks")
        return out.reshape(n, 4)

    def bond_flags(self):
        self._ensure()
        n = lib().mxg_engine_bond_flags(self._e, None, 0)
        out = np.zeros(max(n, 1), dtype=np.uint32)
        check(lib().mxg_engine_bond_flags(self._e, ptr(out, ctypes.c_uint), out.size), "bond_flags")
        return out[:n]

    def space_info(self):
        cdim = np.zeros(3, dtype=np.int32)
        hh = np.zeros(3)
        nc, per = ctypes.c_int(), ctypes.c_uint()
        check(lib().mxg_engine_space_info(self._e, ptr(cdim, ctypes.c_int), ptr(hh, ctypes.c_double),
                                          ctypes.byref(nc), ctypes.byref(per)), "space_info")
        return cdim, hh, nc.value, per.value

    def time_force(self, reps=10):
        self._ensure()
        ms = ctypes.c_double()
        check(lib().mxg_engine_time_force(self._e, int(reps), ctypes.byref(ms)), "time_force")
        return ms.value

    def autotune(self):
        """Picks the force kernel's tile shape and grid by timing candidates on the current
        state; returns the chosen CTAs per SM (force_config() gives the variant and grid)."""
        self._ensure()
        return check(lib().mxg_engine_autotune(self._e), "autotune")

    def force_config(self, variant=None, grid=None):
        """(tile variant, grid) of the force kernel; with both arguments, pins them."""
        self._ensure()
        vv, gg = ctypes.c_int(0 if variant is None else int(variant)), ctypes.c_int(0 if grid is None else int(grid))
        setting = variant is not None and grid is not None
        check(lib().mxg_engine_force_config(self._e, ctypes.byref(vv), ctypes.byref(gg), 1 if setting else 0),
              "force_config")
        return vv.value, gg.value

    def candidate_pairs(self):
        self._ensure()
        c, i = ctypes.c_longlong(), ctypes.c_longlong()
        check(lib().mxg_engine_pair_counts(self._e, ctypes.byref(c), ctypes.byref(i)), "pair_counts")
        return c.value

    def close(self):
        if self._e is not None:
            lib().mxg_engine_finalize(self._e)
            self._e = None


class _UniverseNamespace:
    """``m.Universe``: class-level access to the single universe."""

    def __getattr__(self, name):
        return getattr(universe, name)


# universes holding an engine: finalized at interpreter exit while the CUDA runtime is still up
# (an engine left to the runtime's own teardown can outlive the context its memory belongs to)
_LIVE = weakref.WeakSet()


@atexit.register
def _close_live_universes():
    for u in list(_LIVE):
        try:
            u.close()
        except Exception:
            pass


universe = _Universe()
Universe = _UniverseNamespace()


def _require():
    if universe._e is None:
        raise RuntimeError("mechanica_b200: call init() first")
    return universe


def init(dim=(10.0, 10.0, 10.0), cutoff=1.0, cells=(4, 4, 4), dt=0.01, bc=None, boundary_conditions=None,
         max_distance=None, origin=(0.0, 0.0, 0.0), integrator=FORWARD_EULER, rng="reference", max_types=64,
         stream=None, pair_pruning=0, **ignored):
    """Initialises the universe (MxSimulator_Init / universe_init). Rendering and
    windowing arguments of the reference are accepted and ignored.

    rng: "reference" keeps the reference's deterministic DPD random term
    (dpd_eval.hpp:57); "philox" draws it from a counter-based stream.
    stream: optional CUDA stream handle (int) on which the engine runs.
    pair_pruning: 0 reproduces the reference's sorted-loop pruning (default),
    2 evaluates every pair inside the cutoff (see mxg_engine_set_pair_pruning).
    integrator: FORWARD_EULER or RUNGE_KUTTA_4 (MxSimulator.cpp:218-230)."""
    if integrator not in (FORWARD_EULER, RUNGE_KUTTA_4):
        raise ValueError(f"invalid integrator kind: {integrator}")
    universe.close()
    universe._init(dim, cells, cutoff, dt, bc if bc is not None else boundary_conditions, max_distance, origin,
                   rng, max_types, stream, pair_pruning, integrator)
    return universe


def bind(obj, a, b=None, replica=0):
    return _require().bind(obj, a, b, replica)


def flux(A, B, name, k, decay=0.0):
    """Fickian flux of species `name` between types A and B: k (s_a - s_b) (1 - r/cutoff)^2 per
    pair within the cutoff (MxFluxes_Fick, Flux.cpp:213-227)."""
    _require()._add_flux(0, A, B, name, k, decay, 0.0)


fick = flux


def secrete(A, B, name, k, target, decay=0.0):
    """Secretion of `name` from A to B: max(k (s_a - target), 0) per pair (MxFluxes_Secrete)."""
    _require()._add_flux(1, A, B, name, k, decay, target)


def uptake(A, B, name, k, target, decay=0.0):
    """Uptake of `name` by B from A: max(k (target - s_b) s_a, 0) per pair (MxFluxes_Uptake)."""
    _require()._add_flux(2, A, B, name, k, decay, target)


def step(until=0, dt=0):
    return _require().step(until, dt)


def run(steps=1):
    return _require().steps(steps)
