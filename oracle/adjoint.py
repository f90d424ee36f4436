"""FP64 restatement of the source-free FDTD step, of its transpose and of the
adjoint gradient of a far-field objective.

TEST INFRASTRUCTURE ONLY: the checker of the library's adjoint
(fdtd_adjoint_gradient / fdtd_adjoint_transpose).  The product never imports
it.  It follows the oracle's loops (oracle/fdtd_oracle.c, which restate
yee.c / boundary.c of GSvit) in double precision:

  H half step: ystep_h (yee.c:146-265), then CPML H (boundary.c:347-519 with
               the zero planes of boundary.c:418-492);
  E half step: ystep_e (yee.c:530-1247) with its dispersive branch (the
               Drude + critical-point ADE of yee.c:914-1108 and the CPML inside
               it, yee.c:950-1057, in the reference's own state P^n, P^{n-1},
               E^{n-1}), the PEC rule (yee.c:1138-1237), then CPML E
               (boundary.c:691-884 with the zero planes of boundary.c:522-690).

The TSF corrections are field-independent sources and are left out.  The
coefficients (get_cabs, get_db, the CPML grading) come from the oracle
itself (oracle_get_coeffs / oracle_get_cpml); the far-field series map is
transposed by oracle_farfield_transpose.  The adjoint is checked three ways
in tests/test_adjoint_oracle.py: the forward restatement against the C
oracle, the dot-product identity <M x, y> = <x, M^T y>, and central finite
differences of the objective computed by the C oracle.
"""
import ctypes as C

import numpy as np

from .pyoracle import CpuSolver, _load, series_spectrum

X0, XN, Y0, YN, Z0, ZN = range(6)
EPS0 = 8.854187817620389850e-12
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


def _lib():
    lib, _ = _load("oracle")
    if not getattr(lib, "_adjoint_bound", False):
        lib.oracle_get_coeffs.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, _ip]
        lib.oracle_get_coeffs.restype = C.c_int
        lib.oracle_get_cpml.argtypes = [C.c_void_p, C.c_int] + [_dp] * 6
        lib.oracle_get_cpml.restype = C.c_int
        lib.oracle_farfield_transpose.argtypes = [C.c_void_p, C.c_int, C.c_int, _ip, _dp, _dp]
        lib.oracle_farfield_transpose.restype = C.c_int
        lib.oracle_get_ade_mat.argtypes = [C.c_void_p, _ip]
        lib.oracle_get_ade_mat.restype = C.c_int
        lib._adjoint_bound = True
    return lib


def _p(a):
    return a.ctypes.data_as(_dp)


class LinearStep:
    """The source-free step M of an oracle run and its transpose M^T."""

    def __init__(self, solver: CpuSolver):
        lib = _lib()
        sc = solver.scene
        self.shape = X, Y, Z = sc.xres, sc.yres, sc.zres
        self.dx = sc.dx
        n = X * Y * Z
        ca, cb = np.zeros(3 * n), np.zeros(3 * n)
        da, db = np.zeros(n), np.zeros(n)
        fl = np.zeros(n, dtype=np.int32)
        lib.oracle_get_coeffs(solver.h, _p(ca), _p(cb), _p(da), _p(db), fl.ctypes.data_as(_ip))
        self.ca, self.cb = ca.reshape(3, X, Y, Z), cb.reshape(3, X, Y, Z)
        self.da, self.db = da.reshape(X, Y, Z), db.reshape(X, Y, Z)
        fl = fl.reshape(X, Y, Z)
        self.t = [(fl & (1 << a)) != 0 for a in range(3)]          # tbc: ordinary update
        self.pec = [(fl & (8 << a)) != 0 for a in range(3)]        # zeroed by the PEC rule
        # dispersive branch: the cells, the material whose ADE coefficients they
        # use, per-cell coefficient arrays, and the components it forms
        am = np.zeros(n, dtype=np.int32)
        lib.oracle_get_ade_mat(solver.h, am.ctypes.data_as(_ip))
        am = am.reshape(X, Y, Z)
        self.ade = am >= 0
        self.has_ade = bool(self.ade.any())
        if self.has_ade:
            mats = sc.mats
            def coef(name, idx=None):
                v = np.array([(getattr(m, name)[idx] if idx is not None else getattr(m, name)) for m in mats])
                return np.where(self.ade, v[np.maximum(am, 0)], 0.0)
            self.c0, self.c1, self.c2, self.c3 = (coef(k) for k in ("ade_c0", "ade_c1", "ade_c2", "ade_c3"))
            self.a0, self.a1, self.a2 = (coef(k) for k in ("ade_a0", "ade_a1", "ade_a2"))
            self.bp = [[coef(k, q) for q in range(2)] for k in ("ade_bp0", "ade_bp1", "ade_bp2", "ade_bp3", "ade_bp4")]
            eps, sig = coef("epsilon"), coef("sigma")
            dt = sc.dt
            with np.errstate(divide="ignore", invalid="ignore"):
                self.cba = np.where(self.ade, (dt / eps / self.dx) / (1 + sig * dt / 2 / eps), 0.0)
            ii, jj, kk = np.ogrid[:X, :Y, :Z]
            idx = (ii > 0, jj > 0, kk > 0)
            # the ADE value is formed where the component is dispersive (tbc == 0)
            # and its curl exists (yee.c:914-1108)
            self.go = [self.ade & ~self.t[0] & idx[1] & idx[2], self.ade & ~self.t[1] & idx[0] & idx[2],
                       self.ade & ~self.t[2] & idx[0] & idx[1]]
        self.cp = {}
        res = (X, X, Y, Y, Z, Z)
        for f in range(6):
            arrs = [np.zeros(res[f]) for _ in range(6)]
            d = lib.oracle_get_cpml(solver.h, f, *[_p(a) for a in arrs])
            if d > 0:
                self.cp[f] = (d,) + tuple(a[:d].copy() for a in arrs)   # d, be, ce, bh, ch, ke, kh
        # per-axis kappa with the MAX rule of yee.c:179-203 / 573-592
        def kap(lo, hi, nres, h):
            k = np.ones(nres)
            for f, sign in ((lo, 0), (hi, 1)):
                if f in self.cp:
                    d, arr = self.cp[f][0], self.cp[f][6 if h else 5]
                    if sign == 0:
                        k[:d] = np.maximum(k[:d], arr)
                    else:
                        k[nres - d:] = np.maximum(k[nres - d:], arr)
            return k
        self.kxe, self.kye, self.kze = kap(X0, XN, X, 0)[:, None, None], kap(Y0, YN, Y, 0)[None, :, None], kap(Z0, ZN, Z, 0)[None, None, :]
        self.kxh, self.kyh, self.kzh = kap(X0, XN, X, 1)[:, None, None], kap(Y0, YN, Y, 1)[None, :, None], kap(Z0, ZN, Z, 1)[None, None, :]

    # ------------------------------------------------------------------ state
    def zero_state(self):
        X, Y, Z = self.shape
        sh = {X0: (X, Y, Z), XN: (X, Y, Z), Y0: (X, Y, Z), YN: (X, Y, Z), Z0: (X, Y, Z), ZN: (X, Y, Z)}
        st = {"E": [np.zeros(self.shape) for _ in range(3)], "H": [np.zeros(self.shape) for _ in range(3)],
              "pe": {}, "ph": {}}
        if self.has_ade:   # E^{n-1}, P_D^n, P_D^{n-1}, P_cp^n, P_cp^{n-1} per component
            for key in ("ep", "dp", "dpp"):
                st[key] = [np.zeros(self.shape) for _ in range(3)]
            for key in ("p", "pp"):
                st[key] = [[np.zeros(self.shape) for _ in range(2)] for _ in range(3)]
        for f, c in self.cp.items():
            d = c[0]
            s = (d, Y, Z) if f < 2 else (X, d, Z) if f < 4 else (X, Y, d)
            st["pe"][f] = [np.zeros(s), np.zeros(s)]
            st["ph"][f] = [np.zeros(s), np.zeros(s)]
        return st

    # ---------------------------------------------------------------- forward
    def forward(self, st):
        """One source-free step in place (the oracle's loop order)."""
        X, Y, Z = self.shape
        dx = self.dx
        ex, ey, ez = st["E"]
        hx, hy, hz = st["H"]
        da, db = self.da, self.db
        kxh, kyh, kzh = self.kxh, self.kyh, self.kzh
        r = (slice(None), slice(0, Y - 1), slice(0, Z - 1))
        hx[r] = da[r] * hx[r] + db[r] * ((ey[:, :Y - 1, 1:] - ey[r]) / kzh[:, :, :Z - 1] - (ez[:, 1:, :Z - 1] - ez[r]) / kyh[:, :Y - 1, :])
        r = (slice(0, X - 1), slice(None), slice(0, Z - 1))
        hy[r] = da[r] * hy[r] + db[r] * ((ez[1:, :, :Z - 1] - ez[r]) / kxh[:X - 1] - (ex[:X - 1, :, 1:] - ex[r]) / kzh[:, :, :Z - 1])
        r = (slice(0, X - 1), slice(0, Y - 1), slice(None))
        hz[r] = da[r] * hz[r] + db[r] * ((ex[:X - 1, 1:, :] - ex[r]) / kyh[:, :Y - 1, :] - (ey[1:, :Y - 1, :] - ey[r]) / kxh[:X - 1])
        self._cpml_h(st, ex, ey, ez, hx, hy, hz, forward=True)
        if self.has_ade:
            self._ade(st, forward=True)
        # ystep_e
        kxe, kye, kze = self.kxe, self.kye, self.kze
        ca, cb, t = self.ca, self.cb, self.t
        r = (slice(None), slice(1, Y), slice(1, Z))
        nx = ca[0][r] * ex[r] + cb[0][r] * ((hz[r] - hz[:, :Y - 1, 1:]) / kye[:, 1:, :] - (hy[r] - hy[:, 1:, :Z - 1]) / kze[:, :, 1:])
        ex[r] = np.where(t[0][r], nx, ex[r])
        r = (slice(1, X), slice(None), slice(1, Z))
        ny = ca[1][r] * ey[r] + cb[1][r] * ((hx[r] - hx[1:, :, :Z - 1]) / kze[:, :, 1:] - (hz[r] - hz[:X - 1, :, 1:]) / kxe[1:])
        ey[r] = np.where(t[1][r], ny, ey[r])
        r = (slice(1, X), slice(1, Y), slice(None))
        nz = ca[2][r] * ez[r] + cb[2][r] * ((hy[r] - hy[:X - 1, 1:, :]) / kxe[1:] - (hx[r] - hx[1:, :Y - 1, :]) / kye[:, 1:, :])
        ez[r] = np.where(t[2][r], nz, ez[r])
        for a, e in enumerate((ex, ey, ez)):
            e[self.pec[a]] = 0.0
        self._cpml_e(st, ex, ey, ez, hx, hy, hz, forward=True)

    # ---------------------------------------------------------------- adjoint
    def adjoint(self, ad):
        """The transposed step in place on adjoint state `ad` (same layout)."""
        X, Y, Z = self.shape
        eb, hb = ad["E"], ad["H"]
        ebx, eby, ebz = eb
        hbx, hby, hbz = hb
        # E half step, reversed: CPML corrections and psi_E, zero planes, PEC, ystep_e
        self._cpml_e(ad, ebx, eby, ebz, hbx, hby, hbz, forward=False)
        for a in range(3):
            eb[a][self.pec[a]] = 0.0
        kxe, kye, kze = self.kxe, self.kye, self.kze
        ca, cb, t = self.ca, self.cb, self.t
        r = (slice(None), slice(1, Y), slice(1, Z))
        w = np.where(t[0][r], cb[0][r] * ebx[r], 0.0)
        hbz[r] += w / kye[:, 1:, :]
        hbz[:, :Y - 1, 1:] -= w / kye[:, 1:, :]
        hby[r] -= w / kze[:, :, 1:]
        hby[:, 1:, :Z - 1] += w / kze[:, :, 1:]
        ebx[r] = np.where(t[0][r], ca[0][r] * ebx[r], ebx[r])
        r = (slice(1, X), slice(None), slice(1, Z))
        w = np.where(t[1][r], cb[1][r] * eby[r], 0.0)
        hbx[r] += w / kze[:, :, 1:]
        hbx[1:, :, :Z - 1] -= w / kze[:, :, 1:]
        hbz[r] -= w / kxe[1:]
        hbz[:X - 1, :, 1:] += w / kxe[1:]
        eby[r] = np.where(t[1][r], ca[1][r] * eby[r], eby[r])
        r = (slice(1, X), slice(1, Y), slice(None))
        w = np.where(t[2][r], cb[2][r] * ebz[r], 0.0)
        hby[r] += w / kxe[1:]
        hby[:X - 1, 1:, :] -= w / kxe[1:]
        hbx[r] -= w / kye[:, 1:, :]
        hbx[1:, :Y - 1, :] += w / kye[:, 1:, :]
        ebz[r] = np.where(t[2][r], ca[2][r] * ebz[r], ebz[r])
        if self.has_ade:
            self._ade(ad, forward=False)
        # H half step, reversed: zero planes and CPML H, ystep_h
        self._cpml_h(ad, ebx, eby, ebz, hbx, hby, hbz, forward=False)
        da, db = self.da, self.db
        kxh, kyh, kzh = self.kxh, self.kyh, self.kzh
        r = (slice(None), slice(0, Y - 1), slice(0, Z - 1))
        w = db[r] * hbx[r]
        eby[:, :Y - 1, 1:] += w / kzh[:, :, :Z - 1]
        eby[r] -= w / kzh[:, :, :Z - 1]
        ebz[:, 1:, :Z - 1] -= w / kyh[:, :Y - 1, :]
        ebz[r] += w / kyh[:, :Y - 1, :]
        hbx[r] = da[r] * hbx[r]
        r = (slice(0, X - 1), slice(None), slice(0, Z - 1))
        w = db[r] * hby[r]
        ebz[1:, :, :Z - 1] += w / kxh[:X - 1]
        ebz[r] -= w / kxh[:X - 1]
        ebx[:X - 1, :, 1:] -= w / kzh[:, :, :Z - 1]
        ebx[r] += w / kzh[:, :, :Z - 1]
        hby[r] = da[r] * hby[r]
        r = (slice(0, X - 1), slice(0, Y - 1), slice(None))
        w = db[r] * hbz[r]
        ebx[:X - 1, 1:, :] += w / kyh[:, :Y - 1, :]
        ebx[r] -= w / kyh[:, :Y - 1, :]
        eby[1:, :Y - 1, :] -= w / kxh[:X - 1]
        eby[r] += w / kxh[:X - 1]
        hbz[r] = da[r] * hbz[r]

    # ------------------------------------------------------------------- ADE
    def _curls(self, H):
        """curl H of ystep_e at every cell (zero where it is not formed)."""
        X, Y, Z = self.shape
        hx, hy, hz = H
        kxe, kye, kze = self.kxe, self.kye, self.kze
        cx, cy, cz = np.zeros(self.shape), np.zeros(self.shape), np.zeros(self.shape)
        r = (slice(None), slice(1, Y), slice(1, Z))
        cx[r] = (hz[r] - hz[:, :Y - 1, 1:]) / kye[:, 1:, :] - (hy[r] - hy[:, 1:, :Z - 1]) / kze[:, :, 1:]
        r = (slice(1, X), slice(None), slice(1, Z))
        cy[r] = (hx[r] - hx[1:, :, :Z - 1]) / kze[:, :, 1:] - (hz[r] - hz[:X - 1, :, 1:]) / kxe[1:]
        r = (slice(1, X), slice(1, Y), slice(None))
        cz[r] = (hy[r] - hy[:X - 1, 1:, :]) / kxe[1:] - (hx[r] - hx[1:, :Y - 1, :]) / kye[:, 1:, :]
        return cx, cy, cz

    def _curls_T(self, H, w):
        """Add the transpose of _curls applied to the weights w (3 arrays)."""
        X, Y, Z = self.shape
        hx, hy, hz = H
        kxe, kye, kze = self.kxe, self.kye, self.kze
        r = (slice(None), slice(1, Y), slice(1, Z))
        v = w[0][r]
        hz[r] += v / kye[:, 1:, :]
        hz[:, :Y - 1, 1:] -= v / kye[:, 1:, :]
        hy[r] -= v / kze[:, :, 1:]
        hy[:, 1:, :Z - 1] += v / kze[:, :, 1:]
        r = (slice(1, X), slice(None), slice(1, Z))
        v = w[1][r]
        hx[r] += v / kze[:, :, 1:]
        hx[1:, :, :Z - 1] -= v / kze[:, :, 1:]
        hz[r] -= v / kxe[1:]
        hz[:X - 1, :, 1:] += v / kxe[1:]
        r = (slice(1, X), slice(1, Y), slice(None))
        v = w[2][r]
        hy[r] += v / kxe[1:]
        hy[:X - 1, 1:, :] -= v / kxe[1:]
        hx[r] -= v / kye[:, 1:, :]
        hx[1:, :Y - 1, :] += v / kye[:, 1:, :]

    def _ade_cpml_faces(self):
        """The psi_E updates of the CPML inside the dispersive branch
        (yee.c:950-1057), per face: (face, cells, previous cells along the
        normal, psi cells, (psi index, H component, [(E component, sign)]) ...).
        The x0 corrections are scaled by cb = 0 in the reference and vanish."""
        X, Y, Z = self.shape
        out = []
        for f in (X0, Y0, Z0, XN, YN, ZN):
            if f not in self.cp:
                continue
            d = self.cp[f][0]
            ax = f // 2
            n = (X, Y, Z)[ax]
            lo, hi = (2, d) if f in (X0, Y0, Z0) else (n - d + 1, n)
            if hi <= lo:
                continue
            plo = lo if f in (X0, Y0, Z0) else lo - (n - d)
            cells = [slice(None)] * 3
            cells[ax] = slice(lo, hi)
            prv = list(cells)
            prv[ax] = slice(lo - 1, hi - 1)
            pc = list(cells)
            pc[ax] = slice(plo, plo + hi - lo)
            if ax == 0:
                pairs = ((0, 2, [] if f == X0 else [(1, -1)]), (1, 1, [] if f == X0 else [(2, +1)]))
            elif ax == 1:
                pairs = ((0, 2, [(0, +1)]), (1, 0, [(2, -1)]))
            else:
                pairs = ((1, 0, [(1, +1)]), (0, 1, [(0, -1)]))
            out.append((f, ax, tuple(cells), tuple(prv), tuple(pc), plo, hi - lo, pairs))
        return out

    def _ade(self, st, forward):
        """The dispersive branch of ystep_e (yee.c:914-1108) on the cells that
        take it: the ADE value of the dispersive components, the CPML inside the
        branch, the polarisation recursions and the state shift.  Forward: in
        place on the state.  Adjoint (forward=False): the transpose, on the
        adjoint state (E: adjoint of the E the ordinary update read; ep, dp, dpp,
        p, pp: adjoints of the state after the step on entry, before it on exit)."""
        X, Y, Z = self.shape
        dx = self.dx
        E, H = st["E"], st["H"]
        m = self.ade
        a0, a1, a2, c0, c1, c2, c3 = self.a0, self.a1, self.a2, self.c0, self.c1, self.c2, self.c3
        bp0, bp1, bp2, bp3, bp4 = self.bp
        faces = self._ade_cpml_faces()
        # the corrections' gate: the two other indices > 0 and the component dispersive
        ii, jj, kk = np.ogrid[:X, :Y, :Z]
        pos = (ii > 0, jj > 0, kk > 0)
        def gate(ax, b):
            g = m & ~self.t[b]
            for o in range(3):
                if o != ax:
                    g = g & pos[o]
            return g
        if forward:
            curl = self._curls(H)
            ve = [e.copy() for e in E]
            dp0 = [x.copy() for x in st["dp"]]
            p0 = [[x.copy() for x in y] for y in st["p"]]
            for a in range(3):
                v = (c0 * curl[a] / dx + c1 * (-a0 * st["dpp"][a] + (1 - a1) * st["dp"][a])
                     + c1 * (-bp0[0] * st["pp"][a][0] + (1 - bp1[0]) * st["p"][a][0])
                     + c1 * (-bp0[1] * st["pp"][a][1] + (1 - bp1[1]) * st["p"][a][1])
                     + c2 * st["ep"][a] + c3 * E[a])
                E[a][:] = np.where(self.go[a], v, E[a])
            for f, ax, cells, prv, pc, plo, ln, pairs in faces:
                shp = [1, 1, 1]
                shp[ax] = ln
                be = self.cp[f][1][plo:plo + ln].reshape(shp)
                ce = self.cp[f][2][plo:plo + ln].reshape(shp)
                for q, hc, corr in pairs:
                    p = st["pe"][f][q]
                    p[pc] = np.where(m[cells], be * p[pc] + ce * (H[hc][cells] - H[hc][prv]) / dx, p[pc])
                    for b, sg in corr:
                        E[b][cells] += np.where(gate(ax, b)[cells], sg * dx * self.cba[cells] * p[pc], 0.0)
            for a in range(3):
                st["dp"][a][:] = np.where(m, a0 * st["dpp"][a] + a1 * dp0[a] + a2 * (st["ep"][a] + 2 * ve[a] + E[a]), st["dp"][a])
                for q in range(2):
                    st["p"][a][q][:] = np.where(m, bp0[q] * st["pp"][a][q] + bp1[q] * p0[a][q] + bp2[q] * st["ep"][a]
                                                + bp3[q] * ve[a] + bp4[q] * E[a], st["p"][a][q])
                st["ep"][a][:] = np.where(m, ve[a], st["ep"][a])
                st["dpp"][a][:] = np.where(m, dp0[a], st["dpp"][a])
                for q in range(2):
                    st["pp"][a][q][:] = np.where(m, p0[a][q], st["pp"][a][q])
            return
        # adjoint: lam1 = adjoints of (E1, ep1, dp1, dpp1, p1, pp1) on entry
        lE1 = [np.where(m, E[a], 0.0) for a in range(3)]
        lep1, ldp1, ldpp1 = st["ep"], st["dp"], st["dpp"]
        lp1, lpp1 = st["p"], st["pp"]
        tot = [lE1[a] + a2 * ldp1[a] + bp4[0] * lp1[a][0] + bp4[1] * lp1[a][1] for a in range(3)]
        # CPML inside the branch, reversed face order
        for f, ax, cells, prv, pc, plo, ln, pairs in reversed(faces):
            shp = [1, 1, 1]
            shp[ax] = ln
            be = self.cp[f][1][plo:plo + ln].reshape(shp)
            ce = self.cp[f][2][plo:plo + ln].reshape(shp)
            for q, hc, corr in reversed(pairs):
                p = st["pe"][f][q]
                lam = p[pc].copy()
                for b, sg in corr:
                    lam += np.where(gate(ax, b)[cells], sg * dx * self.cba[cells] * tot[b][cells], 0.0)
                upd = m[cells]
                p[pc] = np.where(upd, be * lam, lam)
                w = np.where(upd, ce * lam / dx, 0.0)
                H[hc][cells] += w
                H[hc][prv] -= w
        lv = [np.where(self.go[a], tot[a], 0.0) for a in range(3)]
        self._curls_T(H, [c0 / dx * lv[a] for a in range(3)])
        for a in range(3):
            pas = np.where(m & ~self.go[a], tot[a], 0.0)   # E1 = E0 where no ADE value is formed
            lE0 = (c3 * lv[a] + pas + 2 * a2 * ldp1[a] + bp3[0] * lp1[a][0] + bp3[1] * lp1[a][1] + lep1[a])
            lep0 = c2 * lv[a] + a2 * ldp1[a] + bp2[0] * lp1[a][0] + bp2[1] * lp1[a][1]
            ldp0 = c1 * (1 - a1) * lv[a] + a1 * ldp1[a] + ldpp1[a]
            ldpp0 = -c1 * a0 * lv[a] + a0 * ldp1[a]
            lp0 = [c1 * (1 - bp1[q]) * lv[a] + bp1[q] * lp1[a][q] + lpp1[a][q] for q in range(2)]
            lpp0 = [-c1 * bp0[q] * lv[a] + bp0[q] * lp1[a][q] for q in range(2)]
            E[a][:] = np.where(m, lE0, E[a])
            st["ep"][a][:] = np.where(m, lep0, 0.0)
            st["dp"][a][:] = np.where(m, ldp0, 0.0)
            st["dpp"][a][:] = np.where(m, ldpp0, 0.0)
            for q in range(2):
                st["p"][a][q][:] = np.where(m, lp0[q], 0.0)
                st["pp"][a][q][:] = np.where(m, lpp0[q], 0.0)

    # ------------------------------------------------------------------ CPML
    def _cpml_h(self, st, ex, ey, ez, hx, hy, hz, forward):
        """cpml_h of the oracle (boundary.c:347-519).  Forward: psi_H update and
        corrections, zero planes.  Adjoint (ex.. are the E adjoints, hx.. the H
        adjoints): zero planes first, then the transposed corrections."""
        X, Y, Z = self.shape
        dx, db = self.dx, self.db
        ph = st["ph"]
        if not forward:
            if XN in self.cp:
                for h in (hx, hy, hz):
                    h[X - 1, 1:Y - 1, 1:Z - 1] = 0.0
            if YN in self.cp:
                for h in (hx, hy, hz):
                    h[1:X - 1, Y - 1, 1:Z - 1] = 0.0
            if ZN in self.cp:
                for h in (hx, hy, hz):
                    h[1:X - 1, 1:Y - 1, Z - 1] = 0.0
        # (face, cells, psi cells, profile index, axis, the E pair, the H pair with signs)
        for f in (X0, Y0, Z0, XN, YN, ZN):
            if f not in self.cp:
                continue
            d, be, ce, bh, ch = self.cp[f][:5]
            if forward and f in (XN, YN, ZN):
                h0 = (slice(X - 1, X), slice(1, Y - 1), slice(1, Z - 1)) if f == XN else \
                     (slice(1, X - 1), slice(Y - 1, Y), slice(1, Z - 1)) if f == YN else \
                     (slice(1, X - 1), slice(1, Y - 1), slice(Z - 1, Z))
                for h in (hx, hy, hz):
                    h[h0] = 0.0
            if f in (X0, Y0, Z0):
                lo, hi, plo = 0, d - 1, 0
            else:
                n = (X, X, Y, Y, Z, Z)[f]
                lo, hi, plo = n - d + 1, n - 1, 1
            if hi <= lo:
                continue
            ax = f // 2
            cells = [slice(1, X - 1), slice(1, Y - 1), slice(1, Z - 1)]
            cells[ax] = slice(lo, hi)
            nxt = list(cells)
            nxt[ax] = slice(lo + 1, hi + 1)
            pc = list(cells)
            pc[ax] = slice(plo, plo + hi - lo)
            cells, nxt, pc = tuple(cells), tuple(nxt), tuple(pc)
            shp = [1, 1, 1]
            shp[ax] = hi - lo
            bh_ = bh[plo:plo + hi - lo].reshape(shp)
            ch_ = ch[plo:plo + hi - lo].reshape(shp)
            dbd = dx * db[cells]
            # psi[0], psi[1]: the E component of each and the H component and sign of its correction
            if ax == 0:
                pairs = ((0, ez, hy, +1), (1, ey, hz, -1))     # phyx <- ez, phzx <- ey
            elif ax == 1:
                pairs = ((0, ez, hx, -1), (1, ex, hz, +1))     # phxy <- ez, phzy <- ex
            else:
                pairs = ((1, ex, hy, -1), (0, ey, hx, +1))     # phyz <- ex, phxz <- ey
            for q, e, h, sg in pairs:
                p = ph[f][q]
                if forward:
                    p[pc] = bh_ * p[pc] + ch_ * (e[nxt] - e[cells]) / dx
                    h[cells] += sg * dbd * p[pc]
                else:
                    tot = p[pc] + sg * dbd * h[cells]
                    p[pc] = bh_ * tot
                    e[nxt] += ch_ * tot / dx
                    e[cells] -= ch_ * tot / dx

    def _cpml_e(self, st, ex, ey, ez, hx, hy, hz, forward):
        """cpml_e of the oracle (boundary.c:691-884).  Forward: zero planes, psi_E
        update and corrections.  Adjoint: transposed corrections, then the zero
        planes."""
        X, Y, Z = self.shape
        dx, cb, t = self.dx, self.cb, self.t
        pe = st["pe"]
        for f in (X0, Y0, Z0, XN, YN, ZN):
            if f not in self.cp:
                continue
            d, be, ce = self.cp[f][:3]
            ax = f // 2
            if forward and f in (X0, Y0, Z0):
                z0 = [slice(None)] * 3
                z0[ax] = slice(0, 1)
                for e in (ex, ey, ez):
                    e[tuple(z0)] = 0.0
            n = (X, X, Y, Y, Z, Z)[f]
            if f in (X0, Y0, Z0):
                lo, hi, plo = 1, d, 1
            else:
                lo, hi, plo = n - d + 1, n, 1
            if hi <= lo:
                continue
            cells = [slice(None)] * 3
            cells[ax] = slice(lo, hi)
            prv = list(cells)
            prv[ax] = slice(lo - 1, hi - 1)
            pc = list(cells)
            pc[ax] = slice(plo, plo + hi - lo)
            cells, prv, pc = tuple(cells), tuple(prv), tuple(pc)
            shp = [1, 1, 1]
            shp[ax] = hi - lo
            be_ = be[plo:plo + hi - lo].reshape(shp)
            ce_ = ce[plo:plo + hi - lo].reshape(shp)
            # gate of the corrections: the two other indices > 0
            g = np.ones((X, Y, Z), dtype=bool)
            for b in range(3):
                if b != ax:
                    idx = [slice(None)] * 3
                    idx[b] = slice(0, 1)
                    g[tuple(idx)] = False
            g = g[cells]
            # psi[q]: the H component it differences, the E component, its sign, the component gate
            if ax == 0:
                pairs = ((0, hz, ey, 1, -1, 1), (1, hy, ez, 2, +1, 2))
            elif ax == 1:
                pairs = ((0, hz, ex, 0, +1, 0), (1, hx, ez, 2, -1, 2))
            else:
                # the ex correction is gated by zt on the z0 face and by xt on the zn face (boundary.c:758-759, 870-871)
                pairs = ((1, hx, ey, 1, +1, 1), (0, hy, ex, 0, -1, 2 if f == Z0 else 0))
            for q, h, e, a, sg, tg in pairs:
                p = pe[f][q]
                gate = g & t[tg][cells]
                if forward:
                    p[pc] = be_ * p[pc] + ce_ * (h[cells] - h[prv]) / dx
                    e[cells] += np.where(gate, sg * dx * cb[a][cells] * p[pc], 0.0)
                else:
                    tot = p[pc] + np.where(gate, sg * dx * cb[a][cells] * e[cells], 0.0)
                    p[pc] = be_ * tot
                    h[cells] += ce_ * tot / dx
                    h[prv] -= ce_ * tot / dx
        if not forward:
            for f, ax in ((X0, 0), (Y0, 1), (Z0, 2)):
                if f in self.cp:
                    z0 = [slice(None)] * 3
                    z0[ax] = slice(0, 1)
                    for e in (ex, ey, ez):
                        e[tuple(z0)] = 0.0


def design_curl(H, box):
    """curl H of the E update at the cells of box (i0,i1,j0,j1,k0,k1), kappa 1."""
    hx, hy, hz = H
    i0, i1, j0, j1, k0, k1 = box
    c = (slice(i0, i1), slice(j0, j1), slice(k0, k1))
    cx = (hz[c] - hz[i0:i1, j0 - 1:j1 - 1, k0:k1]) - (hy[c] - hy[i0:i1, j0:j1, k0 - 1:k1 - 1])
    cy = (hx[c] - hx[i0:i1, j0:j1, k0 - 1:k1 - 1]) - (hz[c] - hz[i0 - 1:i1 - 1, j0:j1, k0:k1])
    cz = (hy[c] - hy[i0 - 1:i1 - 1, j0:j1, k0:k1]) - (hx[c] - hx[i0:i1, j0 - 1:j1 - 1, k0:k1])
    return np.stack([cx, cy, cz])


def objective_value(solver: CpuSolver, obj) -> float:
    """J = sum_t w_t |F(p_t)|^2 of the DFT of the oracle's far-field series."""
    sc = solver.scene
    F = series_spectrum(solver.nfff_series(), sc.nfff["omega"], sc.dt)
    f = obj["freq"]
    return float(sum(w * np.sum(np.abs(F[p, f]) ** 2) for p, w in zip(obj["points"], obj["weights"])))


def gradient(scene, obj, nsteps: int):
    """(J, dJ/d eps_r of the design cells) in FP64: the forward run and the far
    field by the C oracle on the expanded scene, dJ/dE of the far-field series
    by oracle_farfield_transpose, the backward sweep by LinearStep.adjoint, and
    the chain rule through the edge averaging of get_cabs."""
    lib = _lib()
    box = scene.design["box"]
    i0, i1, j0, j1, k0, k1 = box
    abox = (i0, i1 + 1, j0, j1 + 1, k0, k1 + 1)
    xs = scene.expanded()
    sol = CpuSolver(xs)
    L = LinearStep(sol)
    curls = []
    for _ in range(nsteps):
        sol.step(1)
        curls.append(design_curl(sol.fields()[3:], abox))
    sc = xs
    series = sol.nfff_series()
    F = series_spectrum(series, sc.nfff["omega"], sc.dt)
    f = obj["freq"]
    pts = np.ascontiguousarray(obj["points"], dtype=np.int32)
    J = float(sum(w * np.sum(np.abs(F[p, f]) ** 2) for p, w in zip(pts, obj["weights"])))
    nd = series.shape[-1]
    ph = np.exp(-1j * sc.nfff["omega"][f] * sc.dt * np.arange(nd))
    lam = np.zeros_like(series)
    for p, w in zip(pts, obj["weights"]):
        lam[p] = 2.0 * w * np.real(np.conj(F[p, f])[:, None] * ph[None, :])
    lam = np.ascontiguousarray(lam)
    ad = L.zero_state()
    n = sc.ncells
    shape = L.shape
    gcb = np.zeros((3,) + curls[0].shape[1:])
    c = (slice(abox[0], abox[1]), slice(abox[2], abox[3]), slice(abox[4], abox[5]))
    for m in range(nsteps - 1, -1, -1):
        src = np.zeros(3 * n)
        lib.oracle_farfield_transpose(sol.h, m, len(pts), pts.ctypes.data_as(_ip), _p(lam), _p(src))
        src = src.reshape((3,) + shape)
        for a in range(3):
            ad["E"][a] += src[a]
            gcb[a] += ad["E"][a][c] * curls[m][a]
        L.adjoint(ad)
    # chain rule: cb = dt / (eps_avg dx), eps_avg over the cells sharing the edge
    eps = np.full(shape, EPS0)
    for m_i, mt in enumerate(xs.mats):
        eps[xs.mat == m_i] = mt.epsilon
    bnds = sol.map(1)   # FDTD_MAP_BNDS
    grad = np.zeros((i1 - i0, j1 - j0, k1 - k0))
    dt, dx = sc.dt, sc.dx
    sets = (((0, 0, 0), (0, -1, 0), (0, 0, -1), (0, -1, -1)),
            ((0, 0, 0), (-1, 0, 0), (0, 0, -1), (-1, 0, -1)),
            ((0, 0, 0), (-1, 0, 0), (0, -1, 0), (-1, -1, 0)))
    for ii in range(abox[0], abox[1]):
        for jj in range(abox[2], abox[3]):
            for kk in range(abox[4], abox[5]):
                nc = 4 if bnds[ii, jj, kk] > 0 else 1
                for a in range(3):
                    cells = [(ii + o[0], jj + o[1], kk + o[2]) for o in sets[a][:nc]]
                    e = sum(eps[q] for q in cells) / nc
                    w = gcb[a][ii - abox[0], jj - abox[2], kk - abox[4]] * (-dt / (e * e * dx)) / nc * EPS0
                    for q in cells:
                        if i0 <= q[0] < i1 and j0 <= q[1] < j1 and k0 <= q[2] < k1:
                            grad[q[0] - i0, q[1] - j0, q[2] - k0] += w
    return J, grad


def objective_fd(scene, obj, nsteps: int, cells, h: float):
    """Central differences (J(eps + h) - J(eps - h)) / 2h of the oracle's J for
    the design cells `cells` (index triples within the design box)."""
    out = []
    for q in cells:
        vals = []
        for sgn in (+1, -1):
            s2 = _with_eps(scene, q, sgn * h)
            sol = CpuSolver(s2.expanded())
            sol.step(nsteps)
            vals.append(objective_value(sol, obj))
        out.append((vals[0] - vals[1]) / (2 * h))
    return np.asarray(out)


def _with_eps(scene, q, delta):
    import copy
    s = copy.copy(scene)
    d = dict(scene.design)
    e = np.array(d["eps"], dtype=np.float64, copy=True)
    e[tuple(q)] += delta
    d["eps"] = e
    s.design = d
    return s
