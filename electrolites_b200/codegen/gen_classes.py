"""Code generator for the per-angular-momentum-class ERI + J/K kernels.

For every quartet class (li lj | lk ll) with li >= lj, lk >= ll and the bra
pair class >= the ket pair class (55 classes up to f), this writes one CUDA
translation unit under csrc/generated/ holding

  * a `Cls_<li><lj><lk><ll>` struct of straight-line device functions,
    templated on the arithmetic type T (double for the plain form, float for
    the single-precision quartets of the mixed form):
      - `root_acc`: one Rys root's 2D integrals G_d[e][f] (VRR on centres i
        and k, e <= li+lj, f <= lk+ll) and the accumulation of the
        (e0|f0) Cartesian integrals, all in registers (register form);
      - `row_acc`: the accumulation for one runtime e-component given its
        three rows of 2D integrals (team form, rows staged in shared memory);
      - `hrr_bra` / `hrr_ket`: the horizontal transfers (e0| -> (ij| and
        |f0) -> |kl), applied once per contracted quartet;
  * the instantiation of the kernel templates of csrc/jk_kernels.cuh for
    that class, and a host launcher registered in a table.

The arithmetic follows the reference's Rys formulation (roots t^2, c0x, cpx,
b00, b10, b01 recurrences: electrolites/codegen/gen_khigh.py:128-181) with
one structural change: the transfer to the j and l centres is applied after
the primitive and root sums (late HRR) instead of per root and primitive.

Form selection: the register form is used when the (e0|f0) block has at most
REG_MAX elements; otherwise the team form spreads the e-components over the
lanes of a team (16 or 32*k threads) and splits the f-components over warps.
"""
from __future__ import annotations

import os
import sys
from dataclasses import dataclass

REG_MAX = 100         # largest (e0|f0) block kept in one thread's registers
FPART_MAX = 40        # f-components per warp in the team form
LMAX = 3


def ncart(l):
    return (l + 1) * (l + 2) // 2


def comps(l):
    return [(lx, ly, l - lx - ly) for lx in range(l, -1, -1)
            for ly in range(l - lx, -1, -1)]


def cidx(l, c):
    lx, ly, lz = c
    return (l - lx) * (l - lx + 1) // 2 + lz


@dataclass
class Cls:
    li: int
    lj: int
    lk: int
    ll: int

    @property
    def tag(self):
        return f'{self.li}{self.lj}{self.lk}{self.ll}'

    @property
    def lij(self):
        return self.li + self.lj

    @property
    def lkl(self):
        return self.lk + self.ll

    @property
    def nroots(self):
        return (self.lij + self.lkl) // 2 + 1

    def eset(self):
        return [(L, c) for L in range(self.li, self.lij + 1) for c in comps(L)]

    def fset(self):
        return [(L, c) for L in range(self.lk, self.lkl + 1) for c in comps(L)]

    @property
    def ne(self):
        return len(self.eset())

    @property
    def nf(self):
        return len(self.fset())

    @property
    def form(self):
        return 'reg' if self.ne * self.nf <= REG_MAX else 'team'

    # team form geometry
    @property
    def team_lanes(self):          # lanes holding e-components
        return 16 if self.ne <= 16 else 32 * ((self.ne + 31) // 32)

    @property
    def nwf(self):                 # warps (or half-warp teams) over f
        return (self.nf + FPART_MAX - 1) // FPART_MAX

    @property
    def team_threads(self):
        return self.team_lanes * self.nwf

    def fparts(self):
        n = self.nwf
        size = (self.nf + n - 1) // n
        return [(p * size, min(self.nf, (p + 1) * size)) for p in range(n)]


def all_classes(lmax=LMAX):
    pairs = [(a, b) for a in range(lmax + 1) for b in range(a + 1)]
    out = []
    for A in range(len(pairs)):
        for B in range(A + 1):
            li, lj = pairs[A]
            lk, ll = pairs[B]
            out.append((A, B, Cls(li, lj, lk, ll)))
    return out


def pair_class_index(la, lb):
    return la * (la + 1) // 2 + lb


# ----------------------------------------------------------------------
# expression helpers
# ----------------------------------------------------------------------
class Emitter:
    def __init__(self, indent='        '):
        self.lines = []
        self.ind = indent

    def __call__(self, s):
        self.lines.append(self.ind + s)

    def text(self):
        return '\n'.join(self.lines)


def _mul(a, b):
    if a == '1':
        return b
    if b == '1':
        return a
    return f'{a} * {b}'


def _fma(coef, g, rest):
    """coef * g + rest, with g possibly the literal 1."""
    if g == '1':
        return f'({coef} + {rest})'
    return f'fma({coef}, {g}, {rest})'


def _scaled(n, name):
    return name if n == 1 else f'T({n}) * {name}'


def gen_vrr(em, cls, d, zero_one, lij=None, lkl=None):
    """Emit G_d[e][f] for e <= lij, f <= lkl (default: the class's); returns
    dict (e, f) -> expr.  zero_one: the value of G_d[0][0] ('1' for x and
    y, 'wz' for z)."""
    lij = cls.lij if lij is None else lij
    lkl = cls.lkl if lkl is None else lkl
    g = {(0, 0): zero_one}
    for e in range(lij):
        name = f'g{d}_{e + 1}_0'
        t = _mul(f'c0{d}', g[(e, 0)])
        if e > 0:
            t = _fma(_scaled(e, 'b10'), g[(e - 1, 0)], t)
        em(f'const T {name} = {t};')
        g[(e + 1, 0)] = name
    for f in range(lkl):
        for e in range(lij + 1):
            name = f'g{d}_{e}_{f + 1}'
            expr = _mul(f'cp{d}', g[(e, f)])
            if f > 0:
                expr = _fma(_scaled(f, 'b01'), g[(e, f - 1)], expr)
            if e > 0:
                expr = _fma(_scaled(e, 'b00'), g[(e - 1, f)], expr)
            em(f'const T {name} = {expr};')
            g[(e, f + 1)] = name
    return g


def gen_root_acc(cls):
    em = Emitter('    ')
    gx = gen_vrr(em, cls, 'x', '1')
    gy = gen_vrr(em, cls, 'y', '1')
    gz = gen_vrr(em, cls, 'z', 'wz')
    E, F = cls.eset(), cls.fset()
    # products of x and y factors, shared between accumulators
    uses = {}
    for (_, ec) in E:
        for (_, fc) in F:
            key = (ec[0], fc[0], ec[1], fc[1])
            uses[key] = uses.get(key, 0) + 1
    named = {}
    nf = len(F)
    for ie, (_, ec) in enumerate(E):
        for jf, (_, fc) in enumerate(F):
            a = gx[(ec[0], fc[0])]
            b = gy[(ec[1], fc[1])]
            c = gz[(ec[2], fc[2])]
            key = (ec[0], fc[0], ec[1], fc[1])
            if a == '1' and b == '1':
                xy = None
            elif a == '1':
                xy = b
            elif b == '1':
                xy = a
            elif uses[key] > 1:
                if key not in named:
                    nm = f'xy_{key[0]}{key[1]}{key[2]}{key[3]}'
                    em(f'const T {nm} = {a} * {b};')
                    named[key] = nm
                xy = named[key]
            else:
                xy = f'({a} * {b})'
            k = ie * nf + jf
            if xy is None:
                em(f'acc[{k}] += {c};')
            else:
                em(f'acc[{k}] = fma({xy}, {c}, acc[{k}]);')
    return em.text()


def gen_row_acc(cls, f0, f1):
    """acc[f - f0] += gx[fx] * gy[fy] * gz[fz] for f in [f0, f1)."""
    em = Emitter('    ')
    F = cls.fset()
    for jf in range(f0, f1):
        _, fc = F[jf]
        em(f'acc[{jf - f0}] = fma(gx[{fc[0]}] * gy[{fc[1]}], gz[{fc[2]}], acc[{jf - f0}]);')
    return em.text()


def gen_hrr(la, lb, prefix, vec):
    """(a, b) from levels la..la+lb of the input: out[(a*nb + b) * SO] for a
    at level la, b at level lb.  in[k * SI] is ordered level by level (SI, SO:
    strides, 1 for register arrays, NF for a column of a shared-memory block)."""
    em = Emitter('    ')
    off = {}
    o = 0
    for L in range(la, la + lb + 1):
        off[L] = o
        o += ncart(L)
    memo = {}

    def val(L, a, k, b):
        """value of the (a at level L | b at level k) intermediate."""
        key = (L, a, k, b)
        if key in memo:
            return memo[key]
        if k == 0:
            expr = f'in[{off[L] + cidx(L, a)} * SI]'
            memo[key] = expr
            return expr
        # recurse on the first nonzero direction of b
        d = 0 if b[0] > 0 else (1 if b[1] > 0 else 2)
        bm = list(b)
        bm[d] -= 1
        bm = tuple(bm)
        ap = list(a)
        ap[d] += 1
        ap = tuple(ap)
        t1 = val(L + 1, ap, k - 1, bm)
        t2 = val(L, a, k - 1, bm)
        name = f'{prefix}{k}_{L}_{cidx(L, a)}_{cidx(k, b)}'
        em(f'const T {name} = fma({vec}{"xyz"[d]}, {t2}, {t1});')
        memo[key] = name
        return name

    nb = ncart(lb)
    outs = []
    for ia, a in enumerate(comps(la)):
        for ib, b in enumerate(comps(lb)):
            outs.append(f'out[{ia * nb + ib} * SO] = {val(la, a, lb, b)};')
    for s in outs:
        em(s)
    return em.text()


# ----------------------------------------------------------------------
# nuclear gradient: blocks of the (e|f) space accumulated per quartet
# ----------------------------------------------------------------------
def grad_rects(cls):
    """The four (e|f)-space blocks of the gradient kernel, (name, e-levels,
    f-levels, weight): U unweighted (the lowered shells' transfers read it),
    RA / RB / RC weighted by 2 alpha of the primitive of shell i / j / k
    (the raised shells').  d/dA_x g_a = 2 alpha g_{a+1x} - a_x g_{a-1x}."""
    li, lj, lk, ll = cls.li, cls.lj, cls.lk, cls.ll
    lij, lkl = cls.lij, cls.lkl
    return [('U', (max(li - 1, 0), lij), (max(lk - 1, 0), lkl), None),
            ('RA', (li + 1, lij + 1), (lk, lkl), 'wA'),
            ('RB', (li, lij + 1), (lk, lkl), 'wB'),
            ('RC', (li, lij), (lk + 1, lkl + 1), 'wC')]


def _level_set(l0, l1):
    return [(L, c) for L in range(l0, l1 + 1) for c in comps(L)]


def gen_grad_root(cls, only=None):
    """One Rys root's contribution to the four gradient blocks:
    R[fi * NE_R + ei] (+)= w * G_x G_y G_z over the block's components.
    only: one block's name -- that block alone, written to R with weight w
    (the split classes accumulate one block per pass)."""
    em = Emitter('    ')
    lij1, lkl1 = cls.lij + 1, cls.lkl + 1
    rects = grad_rects(cls)
    if only is not None:
        rects = [('R', e, f, None if w is None else 'w') for name, e, f, w in rects if name == only]
        # the recurrences only as far as this block reads them
        lij1 = max(e[1] for _, e, _, _ in rects)
        lkl1 = max(f[1] for _, _, f, _ in rects)
    gx = gen_vrr(em, cls, 'x', '1', lij1, lkl1)
    gy = gen_vrr(em, cls, 'y', '1', lij1, lkl1)
    gz = gen_vrr(em, cls, 'z', 'wz', lij1, lkl1)
    # every (e, f) component pair of any block, once
    members = {}
    for name, (e0, e1), (f0, f1), w in rects:
        E, F = _level_set(e0, e1), _level_set(f0, f1)
        for jf, (_, fc) in enumerate(F):
            for ie, (_, ec) in enumerate(E):
                members.setdefault((ec, fc), []).append((name, jf * len(E) + ie, w))
    xy_named = {}
    n = 0
    for (ec, fc), targets in members.items():
        a = gx[(ec[0], fc[0])]
        b = gy[(ec[1], fc[1])]
        c = gz[(ec[2], fc[2])]
        key = (ec[0], fc[0], ec[1], fc[1])
        if a == '1' and b == '1':
            xy = None
        elif a == '1':
            xy = b
        elif b == '1':
            xy = a
        else:
            if key not in xy_named:
                nm = f'xy{len(xy_named)}'
                em(f'const T {nm} = {a} * {b};')
                xy_named[key] = nm
            xy = xy_named[key]
        pv = f'p{n}'
        n += 1
        em(f'const T {pv} = {c if xy is None else xy + " * " + c};')
        for name, k, w in targets:
            if w is None:
                em(f'{name}[{k}] += {pv};')
            else:
                em(f'{name}[{k}] = fma({w}, {pv}, {name}[{k}]);')
    return em.text()


MD_LMAX = 6              # = JK_MD_LMAX (csrc/jk_mdj.cuh)
# classes whose J-only builds take the McMurchie-Davidson kernel by default
# (the per-class choice measured against the Rys J engine)
MD_DEFAULT = frozenset()

# component pairs up to which grad_root is straight-line code and the class
# takes the per-lane gradient kernel: measured on (H2O)_32 6-31G* UHF, the
# per-lane form beats the per-warp one up to (dp|ds) (421 pairs; (pp|pp)
# 19.5 -> 10.8 ms, (dd|ps) 17.2 -> 11.2 ms) and loses at (dp|pp) (485: 16.1
# -> 19.2 ms)
GRAD_STRAIGHT_MAX = 450
# per-lane classes with more block products than this accumulate one block
# per pass over the primitives (recurrences and roots recomputed per pass):
# with all four blocks live the accumulators spill to local memory, and the
# (dp|ps) kernel moved 56 GB through DRAM per launch on (H2O)_32 6-31G* UHF.
# Measured there: split, (pp|pp) 10.8 -> 6.2 ms, (ds|pp) 18.4 -> 14.5, (dp|ps)
# 17.1 -> 14.6, (dd|ps) 11.2 -> 9.2; but (ds|ps) (102 products) 10.0 -> 19.8
# and (pp|ps) (124) 9.5 -> 13.3, which stay single-pass
GRAD_SPLIT_MIN = 150
# classes within GRAD_STRAIGHT_MAX that take the per-warp form all the same:
# measured per class on (H2O)_32 6-31G* and (H2O)_16 def2-TZVP UHF against
# the split per-lane form, e.g. (dp|ds) 16.3 -> 10.2 ms, (fs|pp) 45.6 ->
# 19.4 ms, (fp|ps) 54.9 -> 38.3 ms (the per-lane form keeps (dp|ps), (ds|ds),
# (fs|ps): 14.5 against 20.2, 5.6 against 9.2, 24.4 against 35.4 ms)
GRAD_WARP = frozenset({'1111', '2011', '2120', '2210', '3011', '3020', '3110'})


def grad_members(cls):
    """The distinct (e, f) component pairs of the four gradient blocks."""
    mem = set()
    for _, (e0, e1), (f0, f1), _ in grad_rects(cls):
        for _, ec in _level_set(e0, e1):
            for _, fc in _level_set(f0, f1):
                mem.add((ec, fc))
    return mem


def gen_grad_struct(cls):
    """Lines inside the class struct for the gradient kernel: block sizes,
    level ranges and offsets, the root accumulation (straight-line code for
    the smaller classes; the larger ones loop, see jk_grad.cuh, which keeps
    their compile time bounded), and the transfers of the shells raised and
    lowered by one."""
    li, lj, lk, ll = cls.li, cls.lj, cls.lk, cls.ll
    lines = []
    rects = grad_rects(cls)
    small = len(grad_members(cls)) <= GRAD_STRAIGHT_MAX and cls.tag not in GRAD_WARP
    split = small and len(grad_members(cls)) > GRAD_SPLIT_MIN
    lines.append(f'    static constexpr bool G_SMALL = {"true" if small else "false"};')
    lines.append(f'    static constexpr bool G_SPLIT = {"true" if split else "false"};')
    lines.append(f'    static constexpr int G_NMEM = {len(grad_members(cls))};   // block products')
    for name, (e0, e1), (f0, f1), _ in rects:
        ne = len(_level_set(e0, e1))
        nf = len(_level_set(f0, f1))
        lines.append(f'    static constexpr int G_{name}_NE = {ne}, G_{name}_NF = {nf};')
        lines.append(f'    static constexpr int G_{name}_E0 = {e0}, G_{name}_E1 = {e1}, '
                     f'G_{name}_F0 = {f0}, G_{name}_F1 = {f1};')
    lines.append(f'    static constexpr int G_NROOTS = {(cls.lij + cls.lkl + 1) // 2 + 1};')
    # offsets into U of the lowered transfers' inputs
    ue0, uf0 = max(li - 1, 0), max(lk - 1, 0)
    def off(l0, l):
        return sum(ncart(x) for x in range(l0, l))
    lines.append(f'    static constexpr int G_U_E_LI = {off(ue0, li)};    // level li in U\'s e range')
    lines.append(f'    static constexpr int G_U_F_LK = {off(uf0, lk)};    // level lk in U\'s f range')
    tpl = 'template <class T> __device__ static __forceinline__ void'
    if small and not split:
        lines.append(f'    {tpl} grad_root(T c0x, T c0y, T c0z, T cpx, T cpy, T cpz, T b00, '
                     'T b10, T b01, T wz, T wA, T wB, T wC, T *U, T *RA, T *RB, T *RC) {')
        lines.append(gen_grad_root(cls))
        lines.append('    }')
    if split:
        for name, _, _, _ in rects:
            lines.append(f'    {tpl} grad_root_{name}(T c0x, T c0y, T c0z, T cpx, T cpy, T cpz, '
                         'T b00, T b10, T b01, T wz, T w, T *R) {')
            lines.append(gen_grad_root(cls, only=name))
            lines.append('    }')
    tpl_s = ('template <class T, int SI = 1, int SO = 1> __device__ static __forceinline__ '
             'void')
    shifts = [('ip', li + 1, lj, 'hbi', 'AB'), ('jp', li, lj + 1, 'hbj', 'AB'),
              ('kp', lk + 1, ll, 'hkk', 'CD')]
    if li > 0:
        shifts.append(('im', li - 1, lj, 'hbm', 'AB'))
    if lj > 0:
        shifts.append(('jm', li, lj - 1, 'hbn', 'AB'))
    if lk > 0:
        shifts.append(('km', lk - 1, ll, 'hkm', 'CD'))
    for tag, la, lb, prefix, vec in shifts:
        args = 'T ABx, T ABy, T ABz' if vec == 'AB' else 'T CDx, T CDy, T CDz'
        lines.append(f'    {tpl_s} hrr_{tag}(const T *in, T *out, {args}) {{')
        lines.append(gen_hrr(la, lb, prefix, vec))
        lines.append('    }')
    return lines


def gen_class_header(cls):
    E = cls.eset()
    tpl = 'template <class T> __device__ static __forceinline__ void'
    lines = [f'struct Cls_{cls.tag} {{',
             f'    static constexpr int LI = {cls.li}, LJ = {cls.lj}, '
             f'LK = {cls.lk}, LL = {cls.ll};',
             f'    static constexpr int LIJ = {cls.lij}, LKL = {cls.lkl}, '
             f'NROOTS = {cls.nroots};',
             f'    static constexpr int NI = {ncart(cls.li)}, NJ = {ncart(cls.lj)}, '
             f'NK = {ncart(cls.lk)}, NL = {ncart(cls.ll)};',
             f'    static constexpr int NE = {cls.ne}, NF = {cls.nf};',
             f'    static constexpr bool REG = {"true" if cls.form == "reg" else "false"};']
    if cls.form == 'team':
        parts = cls.fparts()
        lines.append(f'    static constexpr int TEAM_LANES = {cls.team_lanes}, '
                     f'NWF = {cls.nwf}, TEAM = {cls.team_threads};')
        lines.append(f'    static constexpr int FPART = {parts[0][1] - parts[0][0]};')
        # e-component table: ex, ey, ez per e index
        ex = ', '.join(str(c[0]) for _, c in E)
        ey = ', '.join(str(c[1]) for _, c in E)
        ez = ', '.join(str(c[2]) for _, c in E)
        lines.append(f'    __device__ static __forceinline__ int ex(int e) '
                     f'{{ constexpr int t[NE] = {{{ex}}}; return t[e]; }}')
        lines.append(f'    __device__ static __forceinline__ int ey(int e) '
                     f'{{ constexpr int t[NE] = {{{ey}}}; return t[e]; }}')
        lines.append(f'    __device__ static __forceinline__ int ez(int e) '
                     f'{{ constexpr int t[NE] = {{{ez}}}; return t[e]; }}')
        for p, (f0, f1) in enumerate(parts):
            lines.append(f'    {tpl} row_acc_{p}('
                         'const T *gx, const T *gy, const T *gz, T *acc) {')
            lines.append(gen_row_acc(cls, f0, f1))
            lines.append('    }')
        lines.append('    template <int P, class T> __device__ static __forceinline__ void '
                     'row_acc(const T *gx, const T *gy, const T *gz, T *acc) {')
        for p in range(len(parts)):
            lines.append(f'        if (P == {p}) row_acc_{p}<T>(gx, gy, gz, acc);')
        lines.append('    }')
        lines.append('    template <int P> __device__ static constexpr int fbegin() {')
        lines.append('        return ' + ' '.join(f'P == {p} ? {f0} :' for p, (f0, _) in enumerate(parts)) + ' 0;')
        lines.append('    }')
        lines.append('    template <int P> __device__ static constexpr int fend() {')
        lines.append('        return ' + ' '.join(f'P == {p} ? {f1} :' for p, (_, f1) in enumerate(parts)) + ' 0;')
        lines.append('    }')
    else:
        lines.append('    static constexpr int TEAM_LANES = 1, NWF = 1, TEAM = 1, FPART = NF;')
        lines.append(f'    {tpl} root_acc('
                     'T c0x, T c0y, T c0z, T cpx, T cpy, T cpz, T b00, T b10, T b01, '
                     'T wz, T *acc) {')
        lines.append(gen_root_acc(cls))
        lines.append('    }')
    tpl_s = ('template <class T, int SI = 1, int SO = 1> __device__ static __forceinline__ '
             'void')
    lines.append(f'    {tpl_s} hrr_bra(const T *in, T *out, T ABx, T ABy, T ABz) {{')
    lines.append(gen_hrr(cls.li, cls.lj, 'hb', 'AB'))
    lines.append('    }')
    lines.append(f'    {tpl_s} hrr_ket(const T *in, T *out, T CDx, T CDy, T CDz) {{')
    lines.append(gen_hrr(cls.lk, cls.ll, 'hk', 'CD'))
    lines.append('    }')
    lines += gen_grad_struct(cls)
    lines.append('};')
    return '\n'.join(lines)


def gen_unit(A, B, cls):
    lines = ['// Generated by electrolites_b200/codegen/gen_classes.py -- do not edit.',
             '#include "../jk_kernels.cuh"',
             '',
             gen_class_header(cls),
             '',
             f'JK_DEFINE_CLASS({cls.tag}, {A}, {B})']
    if cls.lk == 0 and cls.ll == 0:
        # (la lb|ss): its bra transfer is the pair class's, for the J engine
        lines.append(f'JK_DEFINE_PAIR({cls.tag})')
    lines.append('')
    return '\n'.join(lines)


def write_all(outdir, lmax=LMAX):
    os.makedirs(outdir, exist_ok=True)
    classes = all_classes(lmax)
    written = []
    for A, B, cls in classes:
        path = os.path.join(outdir, f'class_{cls.tag}.cu')
        src = gen_unit(A, B, cls)
        old = open(path).read() if os.path.exists(path) else None
        if old != src:
            with open(path + '.tmp', 'w') as f:
                f.write(src)
            os.replace(path + '.tmp', path)
        written.append(path)
    # registry: declarations + table in pair-class order
    reg = ['// Generated by electrolites_b200/codegen/gen_classes.py -- do not edit.',
           '#pragma once',
           '#include "../jk_launch.h"']
    for A, B, cls in classes:
        reg.append(f'int jk_launch_{cls.tag}(const ClassArgs &a, const PlanView *views, '
                   'const LaunchCfg &cfg);')
    reg.append(f'#define JK_NCLASSES {len(classes)}')
    reg.append('static const ClassEntry jk_class_table[JK_NCLASSES] = {')
    for A, B, cls in classes:
        form = 0 if cls.form == 'reg' else 1
        # FP32 quartets by default in the register-form classes that run two
        # blocks per SM ((e0|f0) block <= 27; in the larger register-form
        # ones the second (FP32) copy of the quartet code costs more than it
        # saves) and in the team form (FP32 2D integrals in shared memory)
        fp32 = 1 if (cls.form == 'reg' and cls.ne * cls.nf <= 27) or cls.form != 'reg' else 0
        # McMurchie-Davidson J kernel (J-only builds): register-form classes
        # up to JK_MD_LMAX; md_default: the classes where it measured faster
        # than the Rys J engine
        md = 1 if cls.form == 'reg' and cls.li + cls.lj + cls.lk + cls.ll <= MD_LMAX else 0
        md_def = 1 if md and cls.tag in MD_DEFAULT else 0
        reg.append(f'    {{{A}, {B}, {cls.li}, {cls.lj}, {cls.lk}, {cls.ll}, '
                   f'{form}, {1 if cls.form == "reg" else cls.team_threads}, {fp32}, '
                   f'{md}, {md_def}, jk_launch_{cls.tag}}},')
    reg.append('};')
    # J engine: pair transforms per pair class, from the (la lb|ss) units
    pairs = [(A, cls) for A, B, cls in classes if cls.lk == 0 and cls.ll == 0]
    pairs.sort(key=lambda t: t[0])
    for A, cls in pairs:
        reg.append(f'int jk_pair_dens_{cls.tag}(const PairArgs &a, cudaStream_t st);')
        reg.append(f'int jk_pair_post_{cls.tag}(const PairArgs &a, cudaStream_t st);')
    reg.append(f'#define JK_NPAIR_TABLE {len(pairs)}')
    reg.append('static const PairEntry jk_pair_table[JK_NPAIR_TABLE] = {')
    for A, cls in pairs:
        reg.append(f'    {{{A}, {cls.li}, {cls.lj}, {cls.ne}, jk_pair_dens_{cls.tag}, '
                   f'jk_pair_post_{cls.tag}}},')
    reg.append('};')
    with open(os.path.join(outdir, 'class_table.inc.tmp'), 'w') as f:
        f.write('\n'.join(reg) + '\n')
    os.replace(os.path.join(outdir, 'class_table.inc.tmp'),
               os.path.join(outdir, 'class_table.inc'))
    return written


if __name__ == '__main__':
    out = sys.argv[1] if len(sys.argv) > 1 else os.path.join(
        os.path.dirname(os.path.abspath(__file__)), '..', 'csrc', 'generated')
    for p in write_all(out):
        print(p)
