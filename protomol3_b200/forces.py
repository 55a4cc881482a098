"""Host-side mirror of ProtoMol's force plugin surface over the B200 C ABI.

ProtoMol selects a force by name from a ``.conf`` file (``force LennardJones -algorithm
NonbondedCutoff -switchingFunction C2 -switchon 7 -cutoff 8``), builds it through
``ForceFactory::make`` (factory/ForceFactory.cpp:21) and calls
``SystemForce::evaluate(topology, positions, forces, energies)`` once per step
(force/system/SystemForce.h:32-35), with ``forces`` accumulated into (+=) and energies added to
the ScalarStructure slots.  This module keeps those names, argument meanings and error
behaviour:

* ``Topology`` -- the GenericTopology content the path reads (atoms, types, LJ table, exclusions,
  bonds, angles, periodic box); one or several boxes;
* ``ScalarStructure`` -- energies and virial per box, in ProtoMol's slot order;
* ``NonbondedCutoffSystemForce``, ``NonbondedPMEwaldSystemForce``, ``BondedSystemForce`` --
  ``evaluate(topology, positions, forces, energies)``;
* ``ForceFactory.make(definition)`` -- parses the reference's force definition strings; unknown or
  invalid definitions raise ``ValueError`` (ProtoMol reports an error and returns NULL);
* ``Integrator`` -- the device-resident leapfrog / Langevin loop with ``run(n)`` semantics of
  LeapfrogIntegrator::run (integrator/leapfrog/LeapfrogIntegrator.cpp:89-104).

Every computation runs in libpmb200 on the GPU; there is no CPU fallback.
"""
import ctypes as C
import shlex

import numpy as np

from . import _lib as L

PRECISIONS = {"fp64": L.FP64, "mixed": L.MIXED}


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class ScalarStructure:
    """Energies and virial per box (type/ScalarStructure.h:26-54 slot order)."""
    COULOMB, LENNARDJONES, BOND, ANGLE, VIRIAL = L.E_COULOMB, L.E_LJ, L.E_BOND, L.E_ANGLE, L.E_VIRIAL

    def __init__(self, n_boxes=1, virial=False):
        self.table = np.zeros((n_boxes, L.E_STRIDE))
        self.do_virial = virial

    def clear(self):
        self.table[:] = 0.0

    def __getitem__(self, slot):
        return self.table[0, slot] if self.table.shape[0] == 1 else self.table[:, slot]

    def virial(self, box=0):
        return self.table[box, L.E_VIRIAL:L.E_VIRIAL + 9].reshape(3, 3)

    def potential_energy(self):
        return self.table[:, :4].sum(axis=1)


class Topology:
    """One or more periodic boxes.  ``boxes`` are dicts with the keys produced by
    protomol3_b200.waterbox.water_box (charge already scaled by 18.2226123264)."""

    def __init__(self, boxes, precision="mixed"):
        if isinstance(boxes, dict):
            boxes = [boxes]
        self.boxes = boxes
        self.precision = precision
        self._keep = []
        self._sys = None
        self.n_atoms = int(sum(len(b["charge"]) for b in boxes))
        self.n_boxes = len(boxes)

    def _arr(self, v, dt):
        a = np.ascontiguousarray(np.asarray(v, dt).reshape(-1))
        self._keep.append(a)
        return a

    def system(self):
        if self._sys is None:
            descs = (L.BoxDesc * len(self.boxes))()
            for d, b in zip(descs, self.boxes):
                n = len(b["charge"])
                lj = self._arr(b["lj"], np.float64)
                d.n_atoms = n
                d.n_types = int(round((lj.size // 4) ** 0.5))
                d.charge = _p(self._arr(b["charge"], np.float64))
                d.mass = _p(self._arr(b.get("mass", np.ones(n)), np.float64))
                d.type = _p(self._arr(b["type"], np.int32))
                d.molecule = _p(self._arr(b["molecule"], np.int32))
                d.lj = _p(lj)
                ep = self._arr(b.get("excl_pairs", np.zeros((0, 2))), np.int32)
                d.n_excl = ep.size // 2
                d.excl_pairs = _p(ep)
                d.excl_kind = _p(self._arr(b.get("excl_kind", np.full(ep.size // 2, 2)), np.int32))
                bo = self._arr(b.get("bonds", np.zeros((0, 2))), np.int32)
                d.n_bonds = bo.size // 2
                d.bonds = _p(bo)
                d.bond_k = _p(self._arr(b.get("bond_k", np.zeros(0)), np.float64))
                d.bond_r0 = _p(self._arr(b.get("bond_r0", np.zeros(0)), np.float64))
                an = self._arr(b.get("angles", np.zeros((0, 3))), np.int32)
                d.n_angles = an.size // 3
                d.angles = _p(an)
                d.angle_k = _p(self._arr(b.get("angle_k", np.zeros(0)), np.float64))
                d.angle_theta0 = _p(self._arr(b.get("angle_theta0", np.zeros(0)), np.float64))
                d.ub_k = _p(self._arr(b.get("ub_k", np.zeros(d.n_angles)), np.float64))
                d.ub_r0 = _p(self._arr(b.get("ub_r0", np.zeros(d.n_angles)), np.float64))
                for k in range(3):
                    d.box[k] = float(b["box"][k])
                d.coulomb_scaling = float(b.get("coulomb_scaling", 1.0))
            self._sys = L.checked_ptr(L.lib().pmb_system_create(
                C.cast(descs, C.c_void_p), len(self.boxes), PRECISIONS[self.precision]))
        return self._sys

    def set_skin(self, skin):
        L.check(L.lib().pmb_system_set_skin(self.system(), float(skin)))

    def tuning(self):
        """The speed knobs of this system: dict of skin, sort_cell, pair_ctas_per_sm."""
        t = L.Tuning()
        L.check(L.lib().pmb_system_get_tuning(self.system(), C.byref(t)))
        return {"skin": t.skin, "sort_cell": t.sort_cell, "pair_ctas_per_sm": t.pair_ctas_per_sm}

    def set_tuning(self, skin=None, sort_cell=None, pair_ctas_per_sm=None):
        cur = self.tuning()
        t = L.Tuning()
        t.skin = cur["skin"] if skin is None else float(skin)
        t.sort_cell = cur["sort_cell"] if sort_cell is None else float(sort_cell)
        t.pair_ctas_per_sm = cur["pair_ctas_per_sm"] if pair_ctas_per_sm is None else int(pair_ctas_per_sm)
        L.check(L.lib().pmb_system_set_tuning(self.system(), C.byref(t)))

    def set_vacuum(self, on=True):
        """Vacuum boundary conditions for the cutoff forces: the box (edges from
        ``vacuum_box``) stands in for vacuum, and evaluations refuse positions spread over half
        an edge."""
        L.check(L.lib().pmb_system_set_vacuum(self.system(), int(on)))

    def list_builds(self):
        """Neighbour-list builds so far (waits for the system's stream)."""
        n = C.c_longlong(0)
        L.check(L.lib().pmb_system_list_builds(self.system(), C.byref(n)))
        return n.value

    def list_tiles(self):
        """Pair-kernel tiles of the current neighbour list (8 x 32 pair slots each, padding
        included); waits for the system's stream."""
        n = C.c_longlong(0)
        L.check(L.lib().pmb_system_list_tiles(self.system(), C.byref(n)))
        return n.value

    def evaluate_times(self):
        """Host time (ms) of the last host-pointer evaluation: enqueue, wait for the device's
        first results, accumulation into the caller's arrays (a page-locked force array: the
        wait for the device's sum to land in it)."""
        t = np.zeros(3)
        L.check(L.lib().pmb_system_evaluate_times(self.system(), _p(t)))
        return {"enqueue": t[0], "wait_device": t[1], "accumulate": t[2]}

    def set_stream(self, stream_handle):
        L.check(L.lib().pmb_system_set_stream(self.system(), C.c_void_p(stream_handle)))

    def positions(self):
        return np.concatenate([np.asarray(b["pos"], np.float64).reshape(-1, 3) for b in self.boxes])

    def velocities(self):
        return np.concatenate([np.asarray(b["vel"], np.float64).reshape(-1, 3) for b in self.boxes])

    def close(self):
        if self._sys is not None:
            L.lib().pmb_system_destroy(self._sys)
            self._sys = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SystemForce:
    """Base of the B200 forces: ``evaluate(topology, positions, forces, energies)``."""
    keyword = None

    def __init__(self, desc):
        self.desc = desc
        self._handle = None
        self._topo = None

    def handle(self, topo):
        if self._handle is None or self._topo is not topo:
            self._release()
            self._topo = topo
            self._handle = L.checked_ptr(L.lib().pmb_force_create(topo.system(), C.byref(self.desc)))
        return self._handle

    def evaluate(self, topo, positions, forces, energies):
        """forces (N,3) and energies (ScalarStructure) are accumulated into, never overwritten."""
        pos = np.ascontiguousarray(positions, np.float64)
        if pos.shape != (topo.n_atoms, 3) or forces.shape != (topo.n_atoms, 3):
            raise ValueError("positions/forces must be (%d, 3)" % topo.n_atoms)
        f = np.ascontiguousarray(forces)
        L.check(L.lib().pmb_force_evaluate(self.handle(topo), _p(pos), _p(f),
                                           _p(energies.table), int(energies.do_virial)))
        if f is not forces:
            forces[:] = f

    def alpha(self, topo):
        a = C.c_double(0.0)
        L.check(L.lib().pmb_force_alpha(self.handle(topo), C.byref(a)))
        return a.value

    def _release(self):
        if self._handle is not None:
            L.lib().pmb_force_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self._release()
        except Exception:
            pass


class NonbondedCutoffSystemForce(SystemForce):
    """``LennardJones [Coulomb] -algorithm NonbondedCutoff`` with per-potential switching
    (module/NonbondedCutoffForceModule.cpp:40-88)."""
    keyword = "NonbondedCutoff"

    def __init__(self, lj=None, coulomb=None):
        d = L.ForceDesc()
        d.kind = L.FORCE_CUTOFF
        if lj is not None:
            d.lj, d.lj_switch, d.lj_switchon, d.lj_cutoff = 1, L.SWITCH[lj[0]], lj[1], lj[2]
        if coulomb is not None:
            d.coulomb, d.coulomb_switch = 1, L.SWITCH[coulomb[0]]
            d.coulomb_switchon, d.coulomb_cutoff = coulomb[1], coulomb[2]
        super().__init__(d)


class NonbondedPMEwaldSystemForce(SystemForce):
    """``Coulomb -algorithm PMEwald -real -reciprocal -correction -interpolation BSpline
    -gridsize nx ny nz -cutoff rc -order p -accuracy a -alpha a``
    (mdl/interface/force/nonbonded/NonbondedPMEwaldSystemForce.h:1003-1061)."""
    keyword = "PMEwald"

    def __init__(self, gridsize, cutoff, order=4, accuracy=1e-6, alpha=-1.0, real=True,
                 reciprocal=True, correction=True, switching="Cutoff", box_grids=None):
        d = L.ForceDesc()
        d.kind = L.FORCE_PME
        for k in range(3):
            d.grid[k] = int(gridsize[k])
        self._bg = None
        if box_grids is not None:
            self._bg = np.ascontiguousarray(np.asarray(box_grids, np.int32).reshape(-1))
            d.box_grids = _p(self._bg)
        d.order, d.cutoff, d.accuracy, d.alpha = int(order), cutoff, accuracy, alpha
        d.real_switch = L.SWITCH[switching]
        d.real, d.reciprocal, d.correction = int(real), int(reciprocal), int(correction)
        super().__init__(d)


class BondedSystemForce(SystemForce):
    """``force Bond, Angle`` (module/BondedForcesModule.cpp:30-31)."""
    keyword = "Bond, Angle"

    def __init__(self):
        d = L.ForceDesc()
        d.kind = L.FORCE_BONDED
        super().__init__(d)


_HANDLE_ARRAYS = {}


def evaluate_all(topo, force_list, positions, forces, energies):
    """ForceGroup::evaluateSystemForces (force/ForceGroup.cpp:54-70) in one device pass.  The
    per-call Python work is kept small (a cached handle array, no copies of contiguous float64
    arrays): it is part of every step of a host-driven integration."""
    hk = tuple(f.handle(topo) for f in force_list)
    hs = _HANDLE_ARRAYS.get(hk)
    if hs is None:
        if len(_HANDLE_ARRAYS) > 64:
            _HANDLE_ARRAYS.clear()
        hs = _HANDLE_ARRAYS[hk] = (C.c_void_p * len(hk))(*hk)
    pos = positions if (isinstance(positions, np.ndarray) and positions.dtype == np.float64
                        and positions.flags.c_contiguous) else np.ascontiguousarray(positions, np.float64)
    f = forces if forces.flags.c_contiguous else np.ascontiguousarray(forces)
    L.check(L.lib().pmb_evaluate(topo.system(), C.addressof(hs), len(hk), pos.ctypes.data, f.ctypes.data,
                                 energies.table.ctypes.data, int(energies.do_virial)))
    if f is not forces:
        forces[:] = f


def profile(topo, force_list, positions=None, nrep=10, flush_l2=True):
    """Mean device time (ms) per pipeline stage of ``force_list``, measured with CUDA events.
    ``positions`` (N, 3) are uploaded first; None reuses those of the last evaluation."""
    hs = (C.c_void_p * len(force_list))(*[f.handle(topo) for f in force_list])
    ms = np.zeros(32)
    n = C.c_int(0)
    names = C.create_string_buffer(1024)
    pos = None
    if positions is not None:
        pos = np.ascontiguousarray(positions, np.float64)
        if pos.shape != (topo.n_atoms, 3):
            raise ValueError("positions must be (%d, 3)" % topo.n_atoms)
    L.check(L.lib().pmb_profile(topo.system(), _p(pos) if pos is not None else None,
                                C.cast(hs, C.c_void_p), len(force_list), int(nrep), int(flush_l2),
                                _p(ms), 32, C.byref(n), names, 1024))
    return dict(zip(names.value.decode().split(","), ms[:n.value].tolist()))


def fp32_peak():
    """Measured FP32 FMA throughput of the current device in TFLOP/s."""
    t = C.c_double(0.0)
    L.check(L.lib().pmb_fp32_peak(C.byref(t)))
    return t.value


class ForceFactory:
    """Parses ProtoMol force definitions (the text after ``force`` in a .conf file).

    Recognised: ``Bond``/``Angle`` (bonded), ``LennardJones``/``Coulomb`` with
    ``-algorithm NonbondedCutoff`` (and the ``NonbondedCutoffB200`` alias), and ``Coulomb
    -algorithm PMEwald`` (alias ``PMEwaldB200``)."""

    @staticmethod
    def make(definition):
        toks = shlex.split(definition.replace(",", " "))
        if not toks:
            raise ValueError("empty force definition")
        names, i = [], 0
        while i < len(toks) and not toks[i].startswith("-"):
            names.append(toks[i])
            i += 1
        opts, cur = {}, None
        for t in toks[i:]:
            if t.startswith("-") and not _is_number(t):
                cur = t[1:]
                opts.setdefault(cur, [])
            elif cur is None:
                raise ValueError("value without option in %r" % definition)
            else:
                opts[cur].append(t)
        if set(names) <= {"Bond", "Angle"}:
            return BondedSystemForce()
        algo = (opts.get("algorithm") or [None])[0]
        if algo in ("NonbondedCutoff", "NonbondedCutoffB200"):
            sw = opts.get("switchingFunction", [])
            son = [float(v) for v in opts.get("switchon", [])]
            cut = [float(v) for v in opts.get("cutoff", [])]
            pots = [n for n in names if n in ("LennardJones", "Coulomb")]
            if not pots or len(pots) != len(names):
                raise ValueError("unknown potential in %r" % definition)
            spec = {}
            si = oi = 0
            for k, pname in enumerate(pots):
                s = sw[k] if k < len(sw) else (sw[-1] if sw else "Cutoff")
                if s not in ("C1", "C2", "Cutoff"):
                    raise ValueError("unknown switching function %r" % s)
                on = 0.0
                if s == "C2":
                    if oi >= len(son):
                        raise ValueError("C2 needs -switchon")
                    on = son[oi]
                    oi += 1
                if si >= len(cut):
                    raise ValueError("missing -cutoff")
                spec[pname] = (s, on, cut[si])
                si += 1 if si + 1 < len(cut) else 0
            return NonbondedCutoffSystemForce(lj=spec.get("LennardJones"), coulomb=spec.get("Coulomb"))
        if algo in ("PMEwald", "PMEwaldB200"):
            if names != ["Coulomb"]:
                raise ValueError("PMEwald is a Coulomb algorithm")
            g = [int(v) for v in opts.get("gridsize", [])]
            if len(g) != 3:
                raise ValueError("-gridsize nx ny nz required")
            return NonbondedPMEwaldSystemForce(
                g, float(opts["cutoff"][0]), order=int((opts.get("order") or [4])[0]),
                accuracy=float((opts.get("accuracy") or [1e-6])[0]),
                alpha=float((opts.get("alpha") or [-1.0])[0]),
                real="real" in opts or not ({"real", "reciprocal", "correction"} & set(opts)),
                reciprocal="reciprocal" in opts or not ({"real", "reciprocal", "correction"} & set(opts)),
                correction="correction" in opts or not ({"real", "reciprocal", "correction"} & set(opts)),
                switching=(opts.get("switchingFunction") or ["Cutoff"])[0])
        raise ValueError("no B200 force registered for %r" % definition)


def _is_number(t):
    try:
        float(t)
        return True
    except ValueError:
        return False


class Integrator:
    """Device-resident MD: ``run(n)`` has LeapfrogIntegrator::run semantics (or
    StandardIntegrator::run for Langevin); the step is replayed from a CUDA graph."""

    def __init__(self, topo, force_list, timestep=1.0, kind="leapfrog", temperature=300.0,
                 gamma=1.0, seed=1234, use_graph=True):
        self.topo = topo
        self.forces = list(force_list)
        d = L.IntegratorDesc()
        d.kind = L.LEAPFROG if kind == "leapfrog" else L.LANGEVIN
        d.timestep_fs, d.temperature, d.gamma_ps, d.seed = timestep, temperature, gamma, seed
        hs = (C.c_void_p * len(self.forces))(*[f.handle(topo) for f in self.forces])
        self._h = L.checked_ptr(L.lib().pmb_md_create(topo.system(), C.cast(hs, C.c_void_p),
                                                      len(self.forces), C.byref(d)))
        L.check(L.lib().pmb_md_use_graph(self._h, int(use_graph)))

    def set_constraints(self, constraints, shake=True, shake_epsilon=1e-5, shake_max_iter=30,
                        rattle=True, rattle_epsilon=1e-5, rattle_max_iter=30):
        """SHAKE after every drift and RATTLE after every step (``shake``/``rattle`` and their
        ``-epsilon``/``-maxIter`` options of module/ModifierModule.cpp:41-48,106-128) on
        ``constraints`` = (atom1, atom2, rest_length) arrays in the reference's list order, e.g.
        from ``constraints.rattle_shake_constraints``."""
        a1, a2, ln = constraints
        self._con = (np.ascontiguousarray(a1, np.int32), np.ascontiguousarray(a2, np.int32),
                     np.ascontiguousarray(ln, np.float64))
        d = L.ConstraintDesc()
        d.n_constraints = len(self._con[0])
        d.atom1, d.atom2, d.rest_length = (_p(a) for a in self._con)
        d.shake, d.shake_epsilon, d.shake_max_iter = int(shake), shake_epsilon, int(shake_max_iter)
        d.rattle, d.rattle_epsilon, d.rattle_max_iter = int(rattle), rattle_epsilon, int(rattle_max_iter)
        L.check(L.lib().pmb_md_set_constraints(self._h, C.byref(d)))

    def constraint_sweeps(self):
        """(SHAKE, RATTLE) sweeps of the last application; max_iter + 1 means not converged."""
        a, b = C.c_int(0), C.c_int(0)
        L.check(L.lib().pmb_md_constraint_sweeps(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def write_frame(self, traj):
        """Appends the current positions to ``traj`` without stopping the device (an
        asynchronous copy and a writer thread; ``traj.flush()`` waits for the file)."""
        L.check(L.lib().pmb_md_write_frame(self._h, traj.handle()))

    def write_force_frame(self, traj):
        """Appends the forces of the last evaluation to ``traj`` (OutputXYZTrajectoryForce with an
        ``Trajectory.xyz_trajectory``), taken like ``write_frame``."""
        L.check(L.lib().pmb_md_write_force_frame(self._h, traj.handle()))

    def checkpoint(self):
        """Exact snapshot of the resident state: dict of positions, velocities, the neighbour
        list's reference positions and the steps taken since the state was set."""
        n = self.topo.n_atoms
        pos, vel, ref = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros((n, 3))
        step = C.c_longlong(0)
        L.check(L.lib().pmb_md_get_checkpoint(self._h, _p(pos), _p(vel), _p(ref), C.byref(step)))
        return {"positions": pos, "velocities": vel, "list_reference": ref, "step": step.value}

    def restore(self, ckpt, exact=True):
        """Restores ``checkpoint()``'s dict, in this run or another of the same boxes and forces;
        ``exact`` rebuilds the neighbour list at the checkpoint's reference positions, so the run
        continues bit for bit."""
        pos = np.ascontiguousarray(ckpt["positions"], np.float64)
        vel = ckpt.get("velocities")
        vel = None if vel is None else np.ascontiguousarray(vel, np.float64)
        ref = np.ascontiguousarray(ckpt["list_reference"], np.float64) if exact else None
        L.check(L.lib().pmb_md_set_checkpoint(self._h, _p(pos), _p(vel), _p(ref) if ref is not None else None,
                                              int(ckpt.get("step", 0))))

    def set_box_noise(self, seeds=None, steps=None):
        """Per-box Langevin noise streams: ``seeds[b]`` and ``steps[b]``, box b's own step count
        at this moment (None keeps them).  A box's noise depends only on its seed, the atom's
        index within the box and its step count, so a box moved into this run from another
        continues that run's noise."""
        nb = self.topo.n_boxes
        sd = None if seeds is None else np.ascontiguousarray(seeds, np.uint64).reshape(nb)
        st = None if steps is None else np.ascontiguousarray(steps, np.int64).reshape(nb)
        L.check(L.lib().pmb_md_set_box_noise(self._h, _p(sd), _p(st)))

    def box_noise(self):
        """(seeds, steps) of every box's noise stream."""
        nb = self.topo.n_boxes
        sd, st = np.zeros(nb, np.uint64), np.zeros(nb, np.int64)
        L.check(L.lib().pmb_md_get_box_noise(self._h, _p(sd), _p(st)))
        return sd, st

    def write_checkpoint(self, config_path, ident, pos_base, vel_base, names, first_step=0):
        """The reference's checkpoint files (OutputCheckpoint): pos_base<id>.pos and
        vel_base<id>.vel in XYZ form and the checkpoint file ``config_path``."""
        arr = (C.c_char_p * len(names))(*[str(x).encode() for x in names])
        L.check(L.lib().pmb_md_write_checkpoint(self._h, str(config_path).encode(), int(ident), int(first_step),
                                                str(pos_base).encode(), str(vel_base).encode(),
                                                C.cast(arr, C.c_void_p)))

    def set_state(self, positions, velocities=None):
        pos = np.ascontiguousarray(positions, np.float64)
        vel = None if velocities is None else np.ascontiguousarray(velocities, np.float64)
        L.check(L.lib().pmb_md_set_state(self._h, _p(pos), _p(vel)))

    def run(self, n):
        L.check(L.lib().pmb_md_run(self._h, int(n)))

    def state(self):
        n = self.topo.n_atoms
        pos, vel = np.zeros((n, 3)), np.zeros((n, 3))
        L.check(L.lib().pmb_md_get_state(self._h, _p(pos), _p(vel)))
        return pos, vel

    def set_virial(self, on=True):
        """Energies with the virial (forces and RATTLE's constraint terms), ScalarStructure's
        virial() switch."""
        L.check(L.lib().pmb_md_set_virial(self._h, int(on)))

    def time_steps(self, n):
        """Mean device time (ms) of a step over n steps (CUDA events on the system's stream)."""
        ms = C.c_double(0.0)
        L.check(L.lib().pmb_md_time(self._h, int(n), C.byref(ms)))
        return ms.value

    def kernels_per_step(self):
        """Kernel launches of one MD step (the list-rebuild kernels exit at once when no rebuild
        is due)."""
        n = C.c_int(0)
        L.check(L.lib().pmb_md_kernels_per_step(self._h, C.byref(n)))
        return n.value

    def device_bytes(self):
        """Device memory held by this run (system, forces, integrator state), in bytes."""
        b = C.c_ulonglong(0)
        L.check(L.lib().pmb_md_device_bytes(self._h, C.byref(b)))
        return b.value

    def forces_now(self):
        f = np.zeros((self.topo.n_atoms, 3))
        L.check(L.lib().pmb_md_get_forces(self._h, _p(f)))
        return f

    def energies(self):
        e = np.zeros((self.topo.n_boxes, L.E_STRIDE))
        k = np.zeros(self.topo.n_boxes)
        L.check(L.lib().pmb_md_energies(self._h, _p(e), _p(k)))
        return e, k

    def close(self):
        if self._h is not None:
            L.lib().pmb_md_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ewald_reciprocal(topo, positions, forces, energies, alpha=-1.0, accuracy=1e-6):
    """The exact Ewald reciprocal sum (NonbondedFullEwaldSystemForce, reciprocal term only),
    the check path for PME: forces (N, 3) and energies (ScalarStructure) are accumulated into."""
    pos = np.ascontiguousarray(positions, np.float64)
    f = np.ascontiguousarray(forces)
    L.check(L.lib().pmb_ewald_reciprocal(topo.system(), _p(pos), float(alpha), float(accuracy), _p(f),
                                         _p(energies.table), int(energies.do_virial)))
    if f is not forces:
        forces[:] = f


def vacuum_box(positions, margin=0.0):
    """Box edges that make a periodic box stand in for vacuum (VacuumBoundaryConditions):
    2 (extent + margin) + 1 per axis, so no two atoms are half an edge apart."""
    pos = np.ascontiguousarray(positions, np.float64).reshape(-1)
    e = np.zeros(3)
    L.check(L.lib().pmb_vacuum_box(_p(pos), pos.size // 3, float(margin), _p(e)))
    return e


class Trajectory:
    """Trajectory files in the reference's formats: ``Trajectory.dcd`` (``DCDFile``,
    output/OutputDCDTrajectory.cpp; io/DCDTrajectoryWriter.cpp) and ``Trajectory.xyz``
    (``finXYZPosFile``, io/XYZWriter.cpp).  Frames come from host positions (``write``) or from
    a device MD run (``Integrator.write_frame``)."""

    def __init__(self, handle, n_atoms):
        self._h = L.checked_ptr(handle)
        self.n_atoms = n_atoms

    @classmethod
    def dcd(cls, path, n_atoms, timestep=1.0, first_step=0, little_endian=True, comment=""):
        return cls(L.lib().pmb_traj_open_dcd(str(path).encode(), int(n_atoms), float(timestep),
                                             int(first_step), int(little_endian), comment.encode()),
                   n_atoms)

    @classmethod
    def xyz(cls, path, names):
        arr = (C.c_char_p * len(names))(*[str(n).encode() for n in names])
        return cls(L.lib().pmb_traj_open_xyz(str(path).encode(), len(names), C.cast(arr, C.c_void_p)),
                   len(names))

    @classmethod
    def xyz_trajectory(cls, path, names):
        """An XYZ trajectory (XYZTrajectoryWriter: a frame-count line, then the frames), the
        file OutputXYZTrajectoryForce writes forces into."""
        arr = (C.c_char_p * len(names))(*[str(n).encode() for n in names])
        return cls(L.lib().pmb_traj_open_xyz_trajectory(str(path).encode(), len(names), C.cast(arr, C.c_void_p)),
                   len(names))

    def set_minimal_image(self, mass, molecule, pairs, box, origin=(0.0, 0.0, 0.0)):
        """DCD frames in minimal image (OutputDCDTrajectory's minimal-image option): molecules
        whole and their centres of mass in the box around ``origin``; ``pairs`` [m, 2] bonds."""
        self._mi = [np.ascontiguousarray(mass, np.float64), np.ascontiguousarray(molecule, np.int32),
                    np.ascontiguousarray(pairs, np.int32).reshape(-1), np.ascontiguousarray(box, np.float64),
                    np.ascontiguousarray(origin, np.float64)]
        m, mol, pr, bx, org = self._mi
        L.check(L.lib().pmb_traj_set_minimal_image(self._h, _p(m), _p(mol), int(pr.size // 2), _p(pr), _p(bx),
                                                   _p(org)))

    def handle(self):
        return self._h

    def write(self, positions):
        pos = np.ascontiguousarray(positions, np.float64).reshape(-1)
        if pos.size != 3 * self.n_atoms:
            raise ValueError("positions must be [n_atoms, 3]")
        L.check(L.lib().pmb_traj_write_host(self._h, _p(pos)))

    def flush(self):
        L.check(L.lib().pmb_traj_flush(self._h))

    def frames(self):
        n = C.c_longlong(0)
        L.check(L.lib().pmb_traj_frames(self._h, C.byref(n)))
        return n.value

    def close(self):
        if self._h is not None:
            h, self._h = self._h, None
            L.check(L.lib().pmb_traj_close(h))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
