"""ctypes binding of the CPU oracle (oracle/pm_oracle.c) -- test infrastructure only.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline import this module, and only
as the checker.  ``build()`` compiles the C restatement with gcc into oracle/liboracle.so.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

SWITCH = {"cutoff": 0, "C1": 1, "C2": 2}
E_COULOMB, E_LJ, E_BOND, E_ANGLE = 0, 1, 2, 3


def build(force=False):
    src = [os.path.join(HERE, "pm_oracle.c")]
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(s) for s in src + [os.path.join(HERE, "pm_oracle.h")]):
        subprocess.check_call(["gcc", "-O2", "-fPIC", "-shared", "-std=c99", "-o", LIB] + src + ["-lm"])
    return LIB


class OrcSystem(C.Structure):
    _fields_ = [("n", C.c_int), ("ntypes", C.c_int),
                ("charge", C.c_void_p), ("mass", C.c_void_p), ("type", C.c_void_p),
                ("molecule", C.c_void_p), ("lj", C.c_void_p),
                ("nexcl", C.c_int), ("excl_pairs", C.c_void_p), ("excl_kind", C.c_void_p),
                ("nbonds", C.c_int), ("bonds", C.c_void_p), ("bond_k", C.c_void_p),
                ("bond_r0", C.c_void_p), ("nangles", C.c_int), ("angles", C.c_void_p),
                ("angle_k", C.c_void_p), ("angle_theta0", C.c_void_p), ("ub_k", C.c_void_p),
                ("ub_r0", C.c_void_p), ("box", C.c_double * 3), ("coulomb_scaling", C.c_double)]


class OrcCutoff(C.Structure):
    _fields_ = [("do_lj", C.c_int), ("lj_switch", C.c_int), ("lj_switchon", C.c_double),
                ("lj_cutoff", C.c_double), ("do_coul", C.c_int), ("coul_switch", C.c_int),
                ("coul_switchon", C.c_double), ("coul_cutoff", C.c_double)]


class OrcPME(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("order", C.c_int),
                ("cutoff", C.c_double), ("accuracy", C.c_double), ("alpha", C.c_double),
                ("real_switch", C.c_int), ("do_real", C.c_int), ("do_recip", C.c_int),
                ("do_corr", C.c_int)]


class OrcConstraints(C.Structure):
    _fields_ = [("n", C.c_int), ("a1", C.c_void_p), ("a2", C.c_void_p), ("len", C.c_void_p),
                ("shake_eps", C.c_double), ("shake_maxiter", C.c_int),
                ("rattle_eps", C.c_double), ("rattle_maxiter", C.c_int)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(LIB)
        for fn in ("orc_cutoff", "orc_pme", "orc_bonded", "orc_leapfrog",
                   "orc_leapfrog_constrained", "orc_shake", "orc_rattle", "orc_langevin",
                   "orc_langevin_constrained"):
            getattr(_lib, fn).restype = C.c_int
        _lib.orc_pme_alpha.restype = C.c_double
        _lib.orc_pme_alpha.argtypes = [C.c_double, C.c_double]
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class System:
    """Owns contiguous numpy copies of a topology dict (keys as written by the fixtures and by
    protomol3_b200.waterbox) and the matching orc_system struct."""

    def __init__(self, topo):
        n = len(topo["charge"])
        self.n = n
        self.keep = {}

        def arr(key, dtype, default=None, shape=None):
            v = topo.get(key, default)
            a = np.ascontiguousarray(np.asarray(v, dtype=dtype).reshape(-1) if v is not None
                                     else np.zeros(0, dtype))
            self.keep[key] = a
            return a
        lj = arr("lj", np.float64)
        nt = int(round((lj.size // 4) ** 0.5))
        s = OrcSystem()
        s.n = n
        s.ntypes = nt
        s.charge = _p(arr("charge", np.float64))
        s.mass = _p(arr("mass", np.float64, np.ones(n)))
        s.type = _p(arr("type", np.int32))
        s.molecule = _p(arr("molecule", np.int32))
        s.lj = _p(lj)
        ep = arr("excl_pairs", np.int32, np.zeros((0, 2)))
        s.nexcl = ep.size // 2
        s.excl_pairs = _p(ep)
        s.excl_kind = _p(arr("excl_kind", np.int32, np.zeros(0)))
        b = arr("bonds", np.int32, np.zeros((0, 2)))
        s.nbonds = b.size // 2
        s.bonds = _p(b)
        s.bond_k = _p(arr("bond_k", np.float64, np.zeros(0)))
        s.bond_r0 = _p(arr("bond_r0", np.float64, np.zeros(0)))
        a = arr("angles", np.int32, np.zeros((0, 3)))
        s.nangles = a.size // 3
        s.angles = _p(a)
        s.angle_k = _p(arr("angle_k", np.float64, np.zeros(0)))
        s.angle_theta0 = _p(arr("angle_theta0", np.float64, np.zeros(0)))
        s.ub_k = _p(arr("ub_k", np.float64, np.zeros(0)))
        s.ub_r0 = _p(arr("ub_r0", np.float64, np.zeros(0)))
        box = np.asarray(topo["box"], np.float64)
        for k in range(3):
            s.box[k] = box[k]
        s.coulomb_scaling = float(topo.get("coulomb_scaling", 1.0))
        self.s = s


def cutoff_params(lj=None, coul=None):
    """lj / coul: (switch_name, switchon, cutoff) or None."""
    p = OrcCutoff()
    if lj is not None:
        p.do_lj, p.lj_switch, p.lj_switchon, p.lj_cutoff = 1, SWITCH[lj[0]], lj[1], lj[2]
    if coul is not None:
        p.do_coul, p.coul_switch, p.coul_switchon, p.coul_cutoff = 1, SWITCH[coul[0]], coul[1], coul[2]
    return p


def pme_params(grid, cutoff, order=4, accuracy=1e-6, alpha=-1.0, real_switch="cutoff",
               real=True, recip=True, corr=True):
    p = OrcPME()
    p.nx, p.ny, p.nz = grid
    p.order, p.cutoff, p.accuracy, p.alpha = order, cutoff, accuracy, alpha
    p.real_switch = SWITCH[real_switch]
    p.do_real, p.do_recip, p.do_corr = int(real), int(recip), int(corr)
    return p


def evaluate(system, pos, cutoff=None, pme=None, bonded=False, virial=False):
    """Forces (n,3), energies[4] (Coulomb, LJ, bond, angle), virial (9,) for one configuration."""
    L = lib()
    pos = np.ascontiguousarray(pos, np.float64)
    f = np.zeros((system.n, 3))
    e = np.zeros(4)
    v = np.zeros(9)
    vp = _p(v) if virial else None
    terms = np.zeros(5)
    alpha = C.c_double(0.0)
    if bonded:
        L.orc_bonded(C.byref(system.s), _p(pos), _p(f), _p(e), vp)
    if cutoff is not None:
        L.orc_cutoff(C.byref(system.s), _p(pos), C.byref(cutoff), _p(f), _p(e), vp)
    if pme is not None:
        L.orc_pme(C.byref(system.s), _p(pos), C.byref(pme), _p(f), _p(e), vp,
                  C.byref(alpha), _p(terms))
    return f, e, v, {"alpha": alpha.value, "terms": terms}


def leapfrog(system, pos, vel, dt, nsteps, cutoff=None, pme=None, bonded=True):
    L = lib()
    pos = np.ascontiguousarray(pos, np.float64).copy()
    vel = np.ascontiguousarray(vel, np.float64).copy()
    f = np.zeros((system.n, 3))
    e = np.zeros(4)
    L.orc_leapfrog(C.byref(system.s), C.byref(cutoff) if cutoff is not None else None,
                   C.byref(pme) if pme is not None else None, int(bonded), C.c_double(dt),
                   int(nsteps), _p(pos), _p(vel), _p(f), _p(e))
    return pos, vel, f, e


def langevin(system, pos, vel, dt, nsteps, temperature, gamma, seed=1234, first_step=0,
             cutoff=None, pme=None, bonded=True):
    """LangevinLeapfrogIntegrator::run(nsteps) as orc_langevin restates it (temperature in K,
    gamma in 1/ps), with the device's counter-based noise stream; first_step = steps taken since
    the state was set.  Returns pos, vel, forces, energies of the last evaluation."""
    L = lib()
    pos = np.ascontiguousarray(pos, np.float64).copy()
    vel = np.ascontiguousarray(vel, np.float64).copy()
    f = np.zeros((system.n, 3))
    e = np.zeros(4)
    rc = L.orc_langevin(C.byref(system.s), C.byref(cutoff) if cutoff is not None else None,
                        C.byref(pme) if pme is not None else None, int(bonded), C.c_double(dt),
                        C.c_double(temperature), C.c_double(gamma), C.c_ulonglong(seed),
                        C.c_longlong(first_step), int(nsteps), _p(pos), _p(vel), _p(f), _p(e))
    if rc:
        raise ValueError("orc_langevin: gamma > 0 and temperature >= 0")
    return pos, vel, f, e


def gauss3(seed, atom, stream):
    g = np.zeros(3)
    lib().orc_gauss3(C.c_ulonglong(seed), int(atom), C.c_longlong(stream), _p(g))
    return g


def leapfrog_constrained(system, pos, vel, dt, nsteps, constraints, shake=(1e-5, 30),
                         rattle=(1e-5, 30), cutoff=None, pme=None, bonded=False, last_pos=None,
                         rattle_virial=None):
    """LeapfrogIntegrator::run with SHAKE (post-drift) and RATTLE (post-step) as
    orc_leapfrog_constrained restates them.  constraints = (atom1, atom2, rest_length);
    shake / rattle = (epsilon, max_iter) or None.  Returns pos, vel, forces, energies;
    rattle_virial (numpy array of 9) receives the last RATTLE application's virial."""
    L = lib()
    pos = np.ascontiguousarray(pos, np.float64).copy()
    vel = np.ascontiguousarray(vel, np.float64).copy()
    last = pos.copy() if last_pos is None else np.ascontiguousarray(last_pos, np.float64).copy()
    keep = [np.ascontiguousarray(constraints[0], np.int32), np.ascontiguousarray(constraints[1], np.int32),
            np.ascontiguousarray(constraints[2], np.float64)]
    c = OrcConstraints()
    c.n = len(keep[0])
    c.a1, c.a2, c.len = _p(keep[0]), _p(keep[1]), _p(keep[2])
    c.shake_eps, c.shake_maxiter = shake if shake is not None else (0.0, 0)
    c.rattle_eps, c.rattle_maxiter = rattle if rattle is not None else (0.0, 0)
    f = np.zeros((system.n, 3))
    e = np.zeros(4)
    L.orc_leapfrog_constrained(C.byref(system.s), C.byref(cutoff) if cutoff is not None else None,
                               C.byref(pme) if pme is not None else None, int(bonded), C.byref(c),
                               C.c_double(dt), int(nsteps), _p(pos), _p(vel), _p(last), _p(f), _p(e),
                               _p(rattle_virial) if rattle_virial is not None else None)
    return pos, vel, f, e


def langevin_constrained(system, pos, vel, dt, nsteps, constraints, temperature, gamma, seed=1234,
                         first_step=0, shake=(1e-5, 30), rattle=(1e-5, 30), cutoff=None, pme=None,
                         bonded=False, last_pos=None, rattle_virial=None):
    """LangevinLeapfrogIntegrator::run with SHAKE (post-drift) and RATTLE (post-step) as
    orc_langevin_constrained restates them.  Returns pos, vel, forces, energies."""
    L = lib()
    pos = np.ascontiguousarray(pos, np.float64).copy()
    vel = np.ascontiguousarray(vel, np.float64).copy()
    last = pos.copy() if last_pos is None else np.ascontiguousarray(last_pos, np.float64).copy()
    keep = [np.ascontiguousarray(constraints[0], np.int32), np.ascontiguousarray(constraints[1], np.int32),
            np.ascontiguousarray(constraints[2], np.float64)]
    c = OrcConstraints()
    c.n = len(keep[0])
    c.a1, c.a2, c.len = _p(keep[0]), _p(keep[1]), _p(keep[2])
    c.shake_eps, c.shake_maxiter = shake if shake is not None else (0.0, 0)
    c.rattle_eps, c.rattle_maxiter = rattle if rattle is not None else (0.0, 0)
    f = np.zeros((system.n, 3))
    e = np.zeros(4)
    rc = L.orc_langevin_constrained(C.byref(system.s), C.byref(cutoff) if cutoff is not None else None,
                                    C.byref(pme) if pme is not None else None, int(bonded), C.byref(c),
                                    C.c_double(dt), C.c_double(temperature), C.c_double(gamma),
                                    C.c_ulonglong(seed), C.c_longlong(first_step), int(nsteps), _p(pos),
                                    _p(vel), _p(last), _p(f), _p(e),
                                    _p(rattle_virial) if rattle_virial is not None else None)
    if rc:
        raise ValueError("orc_langevin_constrained: gamma > 0 and temperature >= 0")
    return pos, vel, f, e


def pme_alpha(cutoff, accuracy):
    return lib().orc_pme_alpha(cutoff, accuracy)


# ---------------------------------------------------------------------------------------------
# ProtoMol's own force path compiled from the reference sources (oracle/_ref/libpmref.so,
# built by ``make -C oracle ref`` where the reference tree is present).
# ---------------------------------------------------------------------------------------------
REF_LIB = os.path.join(HERE, "_ref", "libpmref.so")


class RefInput(C.Structure):
    _fields_ = [("n", C.c_int), ("ntypes", C.c_int), ("pos", C.c_void_p), ("charge", C.c_void_p),
                ("mass", C.c_void_p), ("type", C.c_void_p), ("molecule", C.c_void_p),
                ("lj", C.c_void_p), ("nexcl", C.c_int), ("excl_pairs", C.c_void_p),
                ("excl_kind", C.c_void_p), ("nbonds", C.c_int), ("bonds", C.c_void_p),
                ("bond_k", C.c_void_p), ("bond_r0", C.c_void_p), ("nangles", C.c_int),
                ("angles", C.c_void_p), ("angle_k", C.c_void_p), ("angle_theta0", C.c_void_p),
                ("ub_k", C.c_void_p), ("ub_r0", C.c_void_p), ("box", C.c_double * 3),
                ("origin", C.c_double * 3), ("cellsize", C.c_double),
                ("coulomb_scaling", C.c_double)]


class RefCutoff(C.Structure):
    _fields_ = OrcCutoff._fields_


class RefPME(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("order", C.c_int),
                ("cutoff", C.c_double), ("accuracy", C.c_double), ("alpha", C.c_double),
                ("real_switch", C.c_int)]


_ref = None


def ref_available():
    return os.path.exists(REF_LIB)


def ref_root():
    """The ProtoMol 3 source tree the checkers compile from: $PROTOMOL3_REF, else the tree's
    location in the build container."""
    return os.environ.get("PROTOMOL3_REF", "/root/reference")


def build_ref(ref_root=None):
    ref_root = ref_root or globals()["ref_root"]()
    if os.path.isdir(ref_root):
        subprocess.check_call(["make", "-s", "-j8", "-C", HERE, "ref", "REF=" + ref_root])
    return ref_available()


def ref_lib():
    global _ref
    if _ref is None:
        _ref = C.CDLL(REF_LIB)
    return _ref


def _ref_input(system, pos, cellsize):
    k = system.keep
    r = RefInput()
    s = system.s
    r.n, r.ntypes = s.n, s.ntypes
    r.pos = _p(pos)
    for name in ("charge", "mass", "type", "molecule", "lj", "excl_pairs", "excl_kind", "bonds",
                 "bond_k", "bond_r0", "angles", "angle_k", "angle_theta0", "ub_k", "ub_r0"):
        setattr(r, name, getattr(s, name))
    r.nexcl, r.nbonds, r.nangles = s.nexcl, s.nbonds, s.nangles
    for q in range(3):
        r.box[q] = s.box[q]
        r.origin[q] = 0.0
    r.cellsize = cellsize
    r.coulomb_scaling = s.coulomb_scaling
    return r


def ref_evaluate(system, pos, cutoff=None, pme=None, bonded=False, virial=False, cellsize=5.0):
    """Same contract as ``evaluate`` but through the reference's own C++ force classes."""
    L = ref_lib()
    pos = np.ascontiguousarray(pos, np.float64)
    r = _ref_input(system, pos, cellsize)
    f = np.zeros((system.n, 3))
    e = np.zeros(4)
    v = np.zeros(9)
    vp = _p(v) if virial else None
    if bonded:
        L.ref_bonded_eval(C.byref(r), _p(f), _p(e), vp)
    if cutoff is not None:
        c = RefCutoff()
        C.memmove(C.byref(c), C.byref(cutoff), C.sizeof(c))
        L.ref_cutoff_eval(C.byref(r), C.byref(c), _p(f), _p(e), vp)
    if pme is not None:
        p = RefPME()
        p.nx, p.ny, p.nz, p.order = pme.nx, pme.ny, pme.nz, pme.order
        p.cutoff, p.accuracy, p.alpha, p.real_switch = pme.cutoff, pme.accuracy, pme.alpha, pme.real_switch
        L.ref_pme_eval(C.byref(r), C.byref(p), _p(f), _p(e), vp)
    return f, e, v


# ProtoMol's own leapfrog integrator with its SHAKE/RATTLE modifiers (oracle/_ref/libpmref_md.so).
REF_MD_LIB = os.path.join(HERE, "_ref", "libpmref_md.so")
_ref_md = None


def ref_md_available():
    return os.path.exists(REF_MD_LIB)


def ref_leapfrog_constrained(system, elem, pos, vel, dt, nsteps, shake=(1e-5, 30),
                             rattle=(1e-5, 30), all_bonds=True, langevin=None, virial=None):
    """The reference run with no force terms: returns pos, vel and the reference's constraint
    list (atom1, atom2, rest_length).  langevin = (temperature, gamma_ps, seed) runs its
    LangevinLeapfrogIntegrator instead of the LeapfrogIntegrator; virial (numpy array of 9)
    receives the virial its energies hold after the run (the last RATTLE's)."""
    global _ref_md
    if _ref_md is None:
        ref_lib()  # its force path library first (the md library links against it)
        _ref_md = C.CDLL(REF_MD_LIB)
    pos = np.ascontiguousarray(pos, np.float64).copy()
    vel = np.ascontiguousarray(vel, np.float64).copy()
    r = _ref_input(system, pos, 5.0)
    el = C.create_string_buffer(elem.encode() if isinstance(elem, str) else bytes(elem))
    cap = 4 * system.n + 16
    cons = np.zeros(3 * cap, np.int32)
    lens = np.zeros(cap)
    ncon = C.c_int(0)
    se, sm = shake if shake is not None else (0.0, 0)
    re_, rm = rattle if rattle is not None else (0.0, 0)
    if langevin is None:
        rc = _ref_md.ref_leapfrog_constrained(
            C.byref(r), el, int(shake is not None), C.c_double(se), int(sm), int(rattle is not None),
            C.c_double(re_), int(rm), int(all_bonds), C.c_double(dt), int(nsteps), _p(pos), _p(vel),
            C.byref(ncon), _p(cons), _p(lens), cap, _p(virial) if virial is not None else None)
    else:
        temp, gam, seed = langevin
        rc = _ref_md.ref_langevin_constrained(
            C.byref(r), el, int(shake is not None), C.c_double(se), int(sm), int(rattle is not None),
            C.c_double(re_), int(rm), int(all_bonds), C.c_double(dt), C.c_double(temp), C.c_double(gam),
            int(seed), int(nsteps), _p(pos), _p(vel), C.byref(ncon), _p(cons), _p(lens), cap,
            _p(virial) if virial is not None else None)
    if rc:
        raise RuntimeError("reference run failed")
    n = min(ncon.value, cap)
    cons = cons[:3 * n].reshape(-1, 3)
    return pos, vel, (cons[:, 0].copy(), cons[:, 1].copy(), lens[:n].copy())


def _ref_md_lib():
    global _ref_md
    if _ref_md is None:
        ref_lib()
        _ref_md = C.CDLL(REF_MD_LIB)
    return _ref_md


def ref_md_run(system, pos, vel, dt, nsteps, cutoff=None, pme=None, bonded=True, langevin=None,
               keep=("energies",), cellsize=5.0):
    """The reference's own LeapfrogIntegrator (or, with langevin = (temperature, gamma_ps,
    seed), its LangevinLeapfrogIntegrator) stepped by run(1) nsteps times, as ProtoMolApp steps it
    with outputfreq 1 (oracle/ref_md.cpp).  Returns a dict with the arrays named in ``keep``:
    energies [nsteps+1, 4] (Coulomb, LJ, bond, angle), pos / vel / forces [nsteps+1, n, 3]; row k
    is the state after k steps (row 0: the initial forces)."""
    L = _ref_md_lib()
    pos = np.ascontiguousarray(pos, np.float64)
    vel = np.ascontiguousarray(vel, np.float64)
    r = _ref_input(system, pos, cellsize)
    c = p = None
    if cutoff is not None:
        c = RefCutoff()
        C.memmove(C.byref(c), C.byref(cutoff), C.sizeof(c))
    if pme is not None:
        p = RefPME()
        p.nx, p.ny, p.nz, p.order = pme.nx, pme.ny, pme.nz, pme.order
        p.cutoff, p.accuracy, p.alpha, p.real_switch = pme.cutoff, pme.accuracy, pme.alpha, pme.real_switch
    out = {"energies": np.zeros((nsteps + 1, 4))}
    for k in ("pos", "vel", "forces"):
        if k in keep:
            out[k] = np.zeros((nsteps + 1, system.n, 3))
    kind, temp, gam, seed = (0, 0.0, 0.0, 0) if langevin is None else (1,) + tuple(langevin)
    rc = L.ref_md_run(C.byref(r), C.byref(c) if c is not None else None,
                      C.byref(p) if p is not None else None, int(bonded), int(kind), C.c_double(dt),
                      C.c_double(temp), C.c_double(gam), int(seed), _p(vel), int(nsteps),
                      _p(out["energies"]), *[_p(out[k]) if k in out else None
                                             for k in ("pos", "vel", "forces")])
    if rc:
        raise RuntimeError("reference MD run failed")
    return out


def ref_write_dcd(path, frames, timestep=1.0, first_step=0):
    """The reference's DCDTrajectoryWriter, opened as OutputDCDTrajectory opens it, writing
    ``frames`` [n_frames, n_atoms, 3]."""
    fr = np.ascontiguousarray(frames, np.float64)
    rc = _ref_md_lib().ref_write_dcd(str(path).encode(), int(fr.shape[1]), int(fr.shape[0]), _p(fr),
                                     C.c_double(timestep), int(first_step))
    if rc:
        raise RuntimeError("reference DCD writer failed")


def ref_write_xyz(path, pos, names):
    """The reference's XYZWriter::write(coords, names)."""
    p = np.ascontiguousarray(pos, np.float64)
    arr = (C.c_char_p * len(names))(*[str(n).encode() for n in names])
    rc = _ref_md_lib().ref_write_xyz(str(path).encode(), len(names), _p(p), arr)
    if rc:
        raise RuntimeError("reference XYZ writer failed")


def ref_write_xyz_trajectory(path, frames, names):
    """The reference's XYZTrajectoryWriter as OutputXYZTrajectoryForce uses it, one write per frame
    of ``frames`` [n_frames, n_atoms, 3]."""
    fr = np.ascontiguousarray(frames, np.float64)
    arr = (C.c_char_p * len(names))(*[str(n).encode() for n in names])
    rc = _ref_md_lib().ref_write_xyz_trajectory(str(path).encode(), int(fr.shape[1]), int(fr.shape[0]), _p(fr), arr)
    if rc:
        raise RuntimeError("reference XYZ trajectory writer failed")


def ref_write_dcd_minimal(path, system, frames, pairs, origin):
    """The reference's minimal-image DCD output (SemiGenericTopology::minimalImage on each frame,
    then DCDTrajectoryWriter), molecules from the system's molecule indices with ``pairs`` [m, 2]
    as their bonded pairs, box origin ``origin``."""
    fr = np.ascontiguousarray(frames, np.float64)
    r = _ref_input(system, np.ascontiguousarray(fr[0]), 5.0)
    for q in range(3):
        r.origin[q] = float(origin[q])
    pr = np.ascontiguousarray(pairs, np.int32)
    rc = _ref_md_lib().ref_write_dcd_minimal(C.byref(r), int(len(pr)), _p(pr), int(fr.shape[0]), _p(fr),
                                             str(path).encode())
    if rc:
        raise RuntimeError("reference minimal-image DCD writer failed")


def ref_write_checkpoint_config(path, ident, step):
    """The reference's CheckpointConfigWriter with its Random and a LeapfrogIntegrator."""
    with _quiet():
        rc = _ref_md_lib().ref_write_checkpoint_config(str(path).encode(), int(ident), int(step))
    if rc:
        raise RuntimeError("reference checkpoint writer failed")


class _quiet:
    """Keeps the reference's report stream (stdout) out of the caller's output."""

    def __enter__(self):
        import sys
        sys.stdout.flush()
        self.fd = os.dup(1)
        os.dup2(2, 1)

    def __exit__(self, *exc):
        import sys
        sys.stdout.flush()
        os.dup2(self.fd, 1)
        os.close(self.fd)


def ref_evaluate_vacuum(system, pos, cutoff, cellsize=5.0):
    """The reference's cutoff forces with VacuumBoundaryConditions (oracle/ref_vacuum.cpp):
    forces (n, 3), energies[4] (Coulomb, LJ, bond, angle), virial (9,)."""
    L = _ref_md_lib()
    pos = np.ascontiguousarray(pos, np.float64)
    r = _ref_input(system, pos, cellsize)
    c = RefCutoff()
    C.memmove(C.byref(c), C.byref(cutoff), C.sizeof(c))
    f = np.zeros((system.n, 3))
    e = np.zeros(4)
    v = np.zeros(9)
    L.ref_cutoff_eval_vacuum(C.byref(r), C.byref(c), _p(f), _p(e), _p(v))
    return f, e, v


def ref_ewald_reciprocal(system, pos, alpha, accuracy, virial=False):
    """The reference's NonbondedFullEwaldSystemForce with only the reciprocal term
    (oracle/ref_ewald.cpp): forces (n, 3), Coulomb energy, virial (9,)."""
    L = _ref_md_lib()
    pos = np.ascontiguousarray(pos, np.float64)
    r = _ref_input(system, pos, 5.0)
    f = np.zeros((system.n, 3))
    e = np.zeros(4)
    v = np.zeros(9)
    L.ref_ewald_reciprocal(C.byref(r), C.c_double(alpha), C.c_double(accuracy), _p(f), _p(e), _p(v), int(virial))
    return f, e[0], v
