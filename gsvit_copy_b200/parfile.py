"""GSvit parameter files (.par) for the stepping path.

Reads the keyword blocks of GSvit's file parser (parse_settings,
settings.c:3822, keyword dispatch settings.c:3865ff) that describe what the
stepping path computes, together with the MEDIUM_VECTOR material file (the
entity loop of plan.c:4183-4330 with scan_material, plan.c:3113-3232), into
a Scene; and writes GSvit's text outputs of that path: OUT_POINT logs
(output.c:636-660) and NFFF_RAMAHI_POINT far-field logs (output.c:1259-1273).

Keywords read: POOL, COMP, DT_MULT, MATMODE_CHECK, MEDIUM_VECTOR,
BOUNDARY_ALL / BOUNDARY_X0..ZN (cpml or none), SOURCE_TSF (file or generated
source types 1-3), TSF_SKIP, NFFF, NFFF_SKIP, NFFF_RAMAHI_POINT,
NFFF_SPHERICAL_AREA, OUT_POINT.  Keywords of the run environment (VERBOSE,
THREADS, GPU, UGPU, GPU_QUERY, OUT_FILE, OUT_IMAGE) are read and ignored.  Any
other keyword -- other sources, boundaries, media, outputs -- is outside the
implemented path and raises ParError naming it.  Material entities: spheres
(4) and voxel boxes (8) of LINEAR (0), LINTAB (1), PEC (10) or ADE (5)
materials.
"""
from __future__ import annotations

import math
import os
import re
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import abi, plan

MU0 = plan.MU0
EPS0 = plan.EPS0
_IGNORED = {"VERBOSE": "int", "THREADS": "int", "GPU": "int", "UGPU": "int", "GPU_QUERY": "int",
            "OUT_FILE": "line", "OUT_IMAGE": "image"}
_FACES = {"BOUNDARY_X0": 0, "BOUNDARY_XN": 1, "BOUNDARY_Y0": 2, "BOUNDARY_YN": 3, "BOUNDARY_Z0": 4, "BOUNDARY_ZN": 5}
_COMPONENTS = {"ex": 0, "ey": 1, "ez": 2, "hx": 3, "hy": 4, "hz": 5, "all": 6}


class ParError(ValueError):
    pass


@dataclass
class PointOutput:
    component: int        # 0-5 one component, 6 all six
    step: int             # 0 = never written (output.c:593)
    cell: tuple
    filename: str


@dataclass
class ParRun:
    scene: plan.Scene
    points: List[PointOutput] = field(default_factory=list)
    far_files: List[Optional[str]] = field(default_factory=list)   # per far point, NFFF_RAMAHI_POINT name
    base: str = "."


class _Tokens:
    """fscanf-style reading: whitespace-separated tokens, or the rest of a line."""

    def __init__(self, text: str):
        self.t = text
        self.p = 0

    def _skip_ws(self):
        while self.p < len(self.t) and self.t[self.p].isspace():
            self.p += 1

    def word(self) -> Optional[str]:
        self._skip_ws()
        if self.p >= len(self.t):
            return None
        m = re.compile(r"\S+").match(self.t, self.p)
        self.p = m.end()
        return m.group(0)

    def int(self, what) -> int:
        w = self.word()
        try:
            return int(w)
        except (TypeError, ValueError):
            raise ParError(f"{what}: expected an integer, got {w!r}")

    def float(self, what) -> float:
        w = self.word()
        try:
            return float(w)
        except (TypeError, ValueError):
            raise ParError(f"{what}: expected a number, got {w!r}")

    def rest_of_line(self) -> str:
        """%100[^\\n\\r] after the previous token (leading blanks of the line kept out)."""
        while self.p < len(self.t) and self.t[self.p] in " \t":
            self.p += 1
        e = self.p
        while e < len(self.t) and self.t[e] not in "\n\r":
            e += 1
        s = self.t[self.p:e].strip()
        self.p = e
        return s

    def next_line_string(self) -> str:
        """fgets of the rest of the keyword line, then %100[^\\n\\r] (MEDIUM_VECTOR, OUT_FILE)."""
        while self.p < len(self.t) and self.t[self.p] not in "\n":
            self.p += 1
        self.p += 1
        return self.rest_of_line()


def _material(tok: _Tokens, dt: float):
    """scan_material, plan.c:3113-3232: ('linear', eps, mu, sigma, sigast) or a
    table material."""
    typ = tok.int("material type")
    if typ in (0, 1):
        eps, mu, sig, sigast = (plan.f32(tok.float("material")) for _ in range(4))
        if typ == 0:
            return ("linear", eps, mu, sig, sigast)
        return ("table", plan._mat(type=abi.MAT_LINTAB, epsilon=eps * EPS0, mu=mu * MU0, sigma=sig, sigast=sigast))
    if typ == 10:
        return ("table", plan.pec_material())
    if typ == 5:
        eps_inf, sigma, wp, nu = (plan.f32(tok.float("ADE material")) for _ in range(4))
        poles = [tuple(plan.f32(tok.float("ADE pole")) for _ in range(4)) for _ in range(2)]
        return ("table", plan.ade_material(eps_inf, sigma, wp, nu, poles, dt))
    raise ParError(f"material type {typ} is outside the implemented path (LINEAR 0, LINTAB 1, ADE 5, PEC 10)")


def _read_vector(path: str, scene: plan.Scene, matmode_check: int):
    """The MEDIUM_VECTOR entity loop (plan.c:4183-4330) for spheres and voxel boxes."""
    tok = _Tokens(open(path).read())
    ents = []
    while True:
        w = tok.word()
        if w is None:
            break
        typ = int(w)
        if typ == 4:
            c = (tok.float("sphere"), tok.float("sphere"), tok.float("sphere"))
            r = tok.float("sphere radius")
            ents.append(("sphere", (c, r), _material(tok, scene.dt)))
        elif typ == 8:
            p = [tok.int("voxel") for _ in range(6)]
            ents.append(("voxel", (tuple(p[:3]), tuple(p[3:])), _material(tok, scene.dt)))
        else:
            raise ParError(f"material entity {typ} is outside the implemented path (sphere 4, voxel 8)")
    # material mode (plan.c:5492-5517 with test_script_file): linear entities
    # decide ELECTRIC / MAGNETIC; table materials alone leave NONE
    is_e = any(m[0] == "linear" and (m[1] != 1 or m[3] != 0) for _, _, m in ents)
    is_m = any(m[0] == "linear" and (m[2] != 1 or m[4] != 0) for _, _, m in ents)
    if not matmode_check:
        mode = abi.MATMODE_FULL
    elif is_e and not is_m:
        mode = abi.MATMODE_ELECTRIC
    elif is_m and not is_e:
        mode = abi.MATMODE_MAGNETIC
    elif not is_e and not is_m:
        mode = abi.MATMODE_NONE
    else:
        mode = abi.MATMODE_FULL
    shape = (scene.xres, scene.yres, scene.zres)
    scene.matmode = mode
    tables = [m[1] for _, _, m in ents if m[0] == "table"]
    scene.mats = [plan.vacuum_material()] if tables else []
    scene.mat = np.zeros(shape, dtype=np.int32) if tables else None
    linear = any(m[0] == "linear" for _, _, m in ents)   # voxel arrays hold the linear entities
    if linear and mode in (abi.MATMODE_ELECTRIC, abi.MATMODE_FULL):
        scene.epsilon = np.full(shape, np.float32(EPS0), dtype=np.float32)
        scene.sigma = np.zeros(shape, dtype=np.float32)
    if linear and mode in (abi.MATMODE_MAGNETIC, abi.MATMODE_FULL):
        scene.mu = np.full(shape, np.float32(MU0), dtype=np.float32)
        scene.sigast = np.zeros(shape, dtype=np.float32)
    for kind, geo, m in ents:
        if m[0] == "table":
            idx = len(scene.mats)
            for q, old in enumerate(scene.mats[1:], 1):
                if bytes(old) == bytes(m[1]):
                    idx = q
                    break
            if idx == len(scene.mats):
                scene.mats.append(m[1])
            targets = [(scene.mat, idx)]
        else:
            _, eps, mu, sig, sigast = m
            targets = []
            if scene.epsilon is not None:
                targets += [(scene.epsilon, np.float32(eps * EPS0)), (scene.sigma, np.float32(sig))]
            if scene.mu is not None:
                targets += [(scene.mu, np.float32(mu * MU0)), (scene.sigast, np.float32(sigast))]
        for arr, val in targets:
            if kind == "voxel":
                plan.voxel_box(arr, geo[0], geo[1], val)
            else:
                plan.sphere_map(arr, geo[0], geo[1], val)


def load_par(path: str) -> ParRun:
    """Scene and outputs of a GSvit parameter file."""
    base = os.path.dirname(os.path.abspath(path))
    tok = _Tokens(open(path).read())
    pool = None
    nsteps = 0
    dtmult = 1.0
    matmode_check = 0
    vector = None
    cpml = {}
    tsf = None
    tsf_skip = [0] * 6
    nfff_box = None
    nfff_skip = {}
    far = []            # (point, filename or None, individual)
    points = []

    def dt_now():
        if pool is None:
            raise ParError("POOL must precede keywords that need the time step")
        return plan.plan_dt(pool[3], pool[4], pool[5], dtmult)

    while True:
        key = tok.word()
        if key is None:
            break
        if key in _IGNORED:
            kind = _IGNORED[key]
            if kind == "int":
                tok.int(key)
            elif kind == "line":
                tok.next_line_string()
            else:   # OUT_IMAGE: component, step, i, j, k, then the rest of the line
                tok.word()
                for _ in range(4):
                    tok.int(key)
                tok.rest_of_line()
        elif key == "POOL":
            pool = [tok.int(key), tok.int(key), tok.int(key), tok.float(key), tok.float(key), tok.float(key)]
        elif key == "COMP":
            nsteps = tok.int(key)
        elif key == "DT_MULT":
            dtmult = tok.float(key)
        elif key == "MATMODE_CHECK":
            matmode_check = tok.int(key)
        elif key == "MEDIUM_VECTOR":
            vector = tok.next_line_string()
        elif key == "BOUNDARY_ALL" or key in _FACES:
            what = tok.word()
            faces = range(6) if key == "BOUNDARY_ALL" else [_FACES[key]]
            if what == "none":
                for f in faces:
                    cpml.pop(f, None)
            elif what == "cpml":
                depth, m = tok.int(key), tok.int(key)
                sigma, a, kappa = tok.float(key), tok.float(key), tok.float(key)
                for f in faces:
                    cpml[f] = (depth, m, sigma, a, kappa)
            else:
                raise ParError(f"{key} {what}: boundary outside the implemented path (cpml, none)")
        elif key == "SOURCE_TSF":
            box = [tok.int(key) for _ in range(6)]
            th, ph, ps = tok.float(key), tok.float(key), tok.float(key)
            typ = tok.int(key)
            if typ == 0:
                src = ("file", tok.rest_of_line())
            elif typ in (1, 2, 3):
                if nsteps == 0:
                    raise ParError("COMP (number of steps) must precede a generated source")
                wl = tok.float(key)
                width = tok.int(key) if typ == 2 else 0
                span = tok.float(key) if typ == 3 else 0.0
                amp = tok.float(key)
                src = ("gen", typ, wl, width, span, amp)
            else:
                raise ParError("unknown source type")
            tsf = dict(box=box, theta=th, phi=ph, psi=ps, src=src)
        elif key == "TSF_SKIP":
            w = tok.word()
            names = ["i0", "in", "j0", "jn", "k0", "kn"]
            if w not in names:
                raise ParError(f"TSF_SKIP {w}")
            tsf_skip[names.index(w)] = 1
        elif key == "NFFF":
            nfff_box = [tok.int(key) for _ in range(6)]
            tok.int(key)
            tok.int(key)      # sumfrom, sumto: not used by the time-domain series
        elif key == "NFFF_SKIP":
            w = tok.word()
            names = ["i0", "in", "j0", "jn", "k0", "kn"]
            if w not in names:
                raise ParError(f"NFFF_SKIP {w}")
            v = [tok.int(key) for _ in range(4)]
            nfff_skip[names.index(w)] = ((v[0], v[1]), (v[2], v[3]))
        elif key == "NFFF_RAMAHI_POINT":
            p = (tok.int(key), tok.int(key), tok.int(key))
            far.append((p, tok.rest_of_line(), 0))
        elif key == "NFFF_SPHERICAL_AREA":
            thr, phr, rad = tok.int(key), tok.int(key), tok.int(key)
            thf, phf, tht, pht = (tok.float(key) for _ in range(4))
            tok.int(key)    # savefile: image outputs are outside the path
            if pool is None:
                raise ParError("POOL must precede NFFF_SPHERICAL_AREA")
            pts = plan.spherical_area(thr, phr, rad, thf, phf, tht, pht, pool[0], pool[1], pool[2])
            for q, p in enumerate(pts):
                far.append((tuple(int(x) for x in p), None, 1 if q else 0))
        elif key == "OUT_POINT":
            comp = tok.word()
            if comp is None or comp.lower() not in _COMPONENTS:
                raise ParError(f"OUT_POINT component {comp!r} outside the implemented path")
            step = tok.int(key)
            cell = (tok.int(key), tok.int(key), tok.int(key))
            points.append(PointOutput(_COMPONENTS[comp.lower()], step, cell, tok.rest_of_line()))
        else:
            raise ParError(f"keyword {key} is outside the implemented path")

    if pool is None:
        raise ParError("no POOL")
    xr, yr, zr, dx, dy, dz = pool
    if not (dx == dy == dz):
        raise ParError("non-cubic cells are outside the implemented path")
    dt = plan.plan_dt(dx, dy, dz, dtmult)
    s = plan.Scene(name=os.path.basename(path), xres=xr, yres=yr, zres=zr, dx=dx, dt=dt, nsteps=nsteps)
    s.mats = []
    s.matmode = abi.MATMODE_FULL if not matmode_check else abi.MATMODE_NONE
    if vector is not None:
        _read_vector(os.path.join(base, vector), s, matmode_check)
    s.cpml = {f: (d, m, plan.cpml_sigma_opt(m, dx) if sg == -1 else sg, kp, a) for f, (d, m, sg, a, kp) in cpml.items()}
    if tsf is not None:
        b = tsf["box"]
        src = tsf["src"]
        if src[0] == "gen":
            _, typ, wl, width, span, amp = src
            if typ != 2:
                raise ParError(f"generated TSF source type {typ}: only the pulse (2) is implemented")
            wave = plan.tsf_pulse(nsteps, wl, width, dt, amp)
        else:
            t2 = _Tokens(open(os.path.join(base, src[1])).read())
            nd = t2.int("TSF source length")
            wave = np.array([(t2.int("TSF source"), t2.float("TSF source"))[1] for _ in range(nd)])
        s.tsf = dict(box=((b[0], b[1], b[2]), (b[3], b[4], b[5])), theta=tsf["theta"], phi=tsf["phi"],
                     psi=tsf["psi"], skip=tsf_skip, wave=wave)
    if nfff_box is not None and far:
        pts = np.asarray([p for p, _, _ in far], dtype=np.int32)
        ind = [i for _, _, i in far]
        ist = plan.nfff_istart(pts, dt, dx, shared=False)
        for q in range(1, len(far)):          # spherical areas share their first point's istart
            if ind[q]:
                ist[q] = ist[q - 1]
        s.nfff = dict(box=((nfff_box[0], nfff_box[1], nfff_box[2]), (nfff_box[3], nfff_box[4], nfff_box[5])),
                      points=pts, istart=ist, omega=np.zeros(0), series=True, skip=nfff_skip)
    s.probes = np.asarray([p.cell for p in points], dtype=np.int32).reshape(-1, 3)
    return ParRun(scene=s, points=points, far_files=[f for _, f, _ in far], base=base)


def write_outputs(run: ParRun, probes: np.ndarray, series: Optional[np.ndarray], steps_done: int, outdir: str) -> List[str]:
    """GSvit's text outputs after `steps_done` steps: point logs (output.c:636-660,
    rows 0 .. steps_done-2 as at the last step) and far-field logs
    (output.c:1259-1273, -F per data index).  Returns the files written."""
    written = []
    for q, p in enumerate(run.points):
        if p.step == 0:
            continue
        path = os.path.join(outdir, p.filename)
        with open(path, "w") as fh:
            for j in range(max(steps_done - 1, 0)):
                v = probes[q, j]
                if p.component == 6:
                    fh.write("%d %g %g %g %g %g %g\n" % (j, v[0], v[1], v[2], v[3], v[4], v[5]))
                else:
                    fh.write("%d %g\n" % (j, v[p.component]))
        written.append(path)
    if series is not None:
        for n, name in enumerate(run.far_files):
            if not name:
                continue
            path = os.path.join(outdir, name)
            with open(path, "w") as fh:
                for i in range(series.shape[-1]):
                    fh.write("%d %g %g %g\n" % (i, -series[n, 0, i], -series[n, 1, i], -series[n, 2, i]))
            written.append(path)
    return written
