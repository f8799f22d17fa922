"""Generate the golden fixtures in tests/golden/ from the reference's own code.

Run here, where the pHyFlow sources exist (they do not travel with the repo):

    make -C oracle ref
    python tests/golden/make_golden.py [--ref PATH]   (default: $PHYFLOW_REFERENCE, else
                                                      ../reference beside the repository)

Sources of truth:
* direct Gauss velocity   - the reference Cython kernel
  (src/cpp/blobs/cython/vv2parGauss_Cython/vv2parGauss_Cython_cpu.pyx), built
  into oracle/_ref/;
* vortex-panel velocity   - the reference Cython panel kernel
  (src/cpp/panels/cython/vortexPanel_Cython/_vortexPanel_Cython_cpu.pyx);
* remesh                  - the reference ``Regrid`` itself
  (src/python/blobs/base/regrid/_regridding.py), imported under Python 3 with
  stub modules for its two pHyFlow imports: ``blobOptions`` (the constant
  M4PRIME_INTERPKERNEL = 0) and ``m4kernel_1d``, which the reference builds
  with boost.python; here its own weight loop
  (_interpolation_kernels_1d.cpp:74-89, extracted and compiled into
  oracle/_ref/libref_m4.so) stands in for it;
* FMM                     - the reference C++ CPU FMM (oracle/_ref/libreffmm.so);
* population control      - the reference ``PopulationControl`` (same module
  as ``Regrid``);
* induced vorticity       - the reference ww2parGauss_C_cpu loop
  (src/cpp/blobs/c/ww2parGauss_C/ww2parGauss_C_cpu.c), built into oracle/_ref/;
* Tutty diffusion         - the reference ``diffusion_tutty``
  (src/python/blobs/base/evolution/_evolution.py), imported the same way with
  a stub for its ``velocity`` import and the reference ``Regrid`` above.

The fixtures are small .npz files; the generating code is this script.
"""
import argparse
import ast
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "phyflow2.0_b200"))

import oracle  # noqa: E402
from oracle import ref  # noqa: E402
from pfblob import workloads as wl  # noqa: E402


def _py2_module(path, name, env, source=None):
    """Compile a Python-2 module of the reference (or `source`, a part of it)
    with `/` between ints as floor division (Python 2 semantics); nothing else
    is changed."""
    tree = ast.parse(open(path).read() if source is None else source, filename=path)

    class Py2Div(ast.NodeTransformer):
        def visit_BinOp(self, node):
            self.generic_visit(node)
            if isinstance(node.op, ast.Div):
                return ast.copy_location(ast.Call(func=ast.Name("_py2div", ast.Load()),
                                                  args=[node.left, node.right], keywords=[]), node)
            return node

    tree = ast.fix_missing_locations(Py2Div().visit(tree))
    mod = types.ModuleType(name)
    mod.__file__ = path
    mod._py2div = lambda a, b: a // b if (isinstance(a, int) and isinstance(b, int)) else a / b
    mod.__dict__.update(env)
    exec(compile(tree, path, "exec"), mod.__dict__)
    return mod


def load_reference_tutty(refroot):
    """The reference diffusion_tutty, compiled from its own source lines in
    _evolution.py (the rest of that module has Python-2 print statements; this
    function uses only numpy and scipy.sparse)."""
    import scipy
    import scipy.sparse  # noqa: F401
    path = os.path.join(refroot, "src/python/blobs/base/evolution/_evolution.py")
    lines = open(path).read().split("\n")
    a = next(i for i, ln in enumerate(lines) if ln.startswith("def diffusion_tutty("))
    b = next(i for i in range(a + 1, len(lines)) if lines[i].startswith("def "))
    mod = _py2_module(path, "ref_tutty", {"numpy": np, "scipy": scipy},
                      source="\n".join(lines[a:b]))
    return mod.diffusion_tutty


def load_reference_regrid(refroot):
    """Import the reference _regridding.py with stub pHyFlow modules."""
    pk = types.ModuleType("pHyFlow")
    blobs = types.ModuleType("pHyFlow.blobs")
    opts = types.ModuleType("pHyFlow.blobs.blobOptions")
    opts.M4PRIME_INTERPKERNEL = 0
    blobs.blobOptions = opts
    cpp = types.ModuleType("pHyFlow.cpp")
    cppb = types.ModuleType("pHyFlow.cpp.blobs")
    rem = types.ModuleType("pHyFlow.cpp.blobs.remesh")
    if not ref.m4_available():
        raise SystemExit("oracle/_ref/libref_m4.so missing: run `make -C oracle ref` first")
    rem.m4kernel_1d = lambda x, c: ref.m4kernel_1d(x, c)
    rem.__all__ = ["m4kernel_1d"]
    for name, mod in [("pHyFlow", pk), ("pHyFlow.blobs", blobs), ("pHyFlow.blobs.blobOptions", opts),
                      ("pHyFlow.cpp", cpp), ("pHyFlow.cpp.blobs", cppb),
                      ("pHyFlow.cpp.blobs.remesh", rem)]:
        sys.modules[name] = mod
    path = os.path.join(refroot, "src/python/blobs/base/regrid/_regridding.py")
    # The module is Python 2 code: `/` between two ints is floor division
    # there (``kernelSize/2`` at :201-218).  Compile it with every `/` routed
    # through a helper with Python 2 semantics; nothing else is changed.
    tree = ast.parse(open(path).read(), filename=path)

    class Py2Div(ast.NodeTransformer):
        def visit_BinOp(self, node):
            self.generic_visit(node)
            if isinstance(node.op, ast.Div):
                return ast.copy_location(ast.Call(func=ast.Name("_py2div", ast.Load()),
                                                  args=[node.left, node.right], keywords=[]), node)
            return node

    tree = ast.fix_missing_locations(Py2Div().visit(tree))
    mod = types.ModuleType("ref_regridding")
    mod.__file__ = path
    mod._py2div = lambda a, b: a // b if (isinstance(a, int) and isinstance(b, int)) else a / b
    exec(compile(tree, path, "exec"), mod.__dict__)
    return mod


def rand_blobs(n, sigma, seed, lo=0.0, hi=1.0):
    rng = np.random.Generator(np.random.PCG64(seed))
    x = rng.uniform(lo, hi, n)
    y = rng.uniform(lo, hi, n)
    g = rng.standard_normal(n) / n
    return x, y, g, sigma


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get(
        "PHYFLOW_REFERENCE", os.path.join(os.path.dirname(ROOT), "reference")))
    ap.add_argument("--only", choices=["popctl", "tutty", "vorticity", "influence", "regrid",
                                       "cutoff", "source"],
                    default=None,
                    help="write only this group of fixtures")
    args = ap.parse_args()
    if args.only == "popctl":
        population_control_fixtures(args.ref)
        return
    if args.only == "tutty":
        tutty_fixtures(args.ref)
        return
    if args.only == "vorticity":
        vorticity_fixtures()
        return
    if args.only == "influence":
        influence_fixtures()
        return
    if args.only == "cutoff":
        cutoff_fixtures()
        return
    if args.only == "source":
        source_panel_fixtures()
        return
    if args.only == "regrid":  # M4' sweep, Regrid and Tutty fixtures
        regrid_fixtures(args.ref)
        tutty_fixtures(args.ref)
        return
    assert ref.available(), "build oracle/_ref first: make -C oracle ref"

    # 1. direct Gauss, C1 Lamb-Oseen lattice (N = 10 000)
    c1 = wl.lamb_oseen_lattice()
    vx, vy = ref.direct_gauss(c1.x, c1.y, c1.g, c1.ksigmasqr)
    np.savez_compressed(os.path.join(HERE, "direct_c1.npz"), x=c1.x, y=c1.y, g=c1.g,
                        ksigmasqr=c1.ksigmasqr, sigma=c1.sigma, vx=vx, vy=vy)

    # 2. direct Gauss, random blobs with edge cases: a duplicated blob (r = 0
    #    between distinct blobs, EPS path), a zero-circulation blob, a far blob
    x, y, g, sigma = rand_blobs(3000, 0.01, 7)
    x[10], y[10] = x[11], y[11]
    g[20] = 0.0
    x[30], y[30] = 25.0, -13.0
    k2 = 2.0 * sigma * sigma
    vx, vy = ref.direct_gauss(x, y, g, k2)
    np.savez_compressed(os.path.join(HERE, "direct_rand.npz"), x=x, y=y, g=g, ksigmasqr=k2,
                        sigma=sigma, vx=vx, vy=vy)

    # 3. vortex panels: 64 panels on the unit cylinder, targets around it,
    #    including points on a panel line extension and very close to panels
    ps = wl.cylinder_panels(64, config=3, instance=7)
    rng = np.random.Generator(np.random.PCG64(11))
    r = rng.uniform(1.0005, 3.0, 2000)
    t = rng.uniform(-np.pi, np.pi, 2000)
    xv = r * np.cos(t)
    yv = r * np.sin(t)
    # points on the extension of panel 0 and right next to its midpoint
    dx, dy = ps.xe[0] - ps.xs[0], ps.ye[0] - ps.ys[0]
    xv[:3] = ps.xe[0] + dx * np.array([0.5, 1.0, 3.0])
    yv[:3] = ps.ye[0] + dy * np.array([0.5, 1.0, 3.0])
    xv[3] = 0.5 * (ps.xs[0] + ps.xe[0]) - 1e-6 * dy
    yv[3] = 0.5 * (ps.ys[0] + ps.ye[0]) + 1e-6 * dx
    vx, vy = ref.panel_velocity(ps.gamma, ps.xs, ps.ys, ps.xe, ps.ye, ps.cosa, ps.sina, xv, yv)
    np.savez_compressed(os.path.join(HERE, "panel_cyl.npz"), gamma=ps.gamma, xs=ps.xs, ys=ps.ys,
                        xe=ps.xe, ye=ps.ye, cosa=ps.cosa, sina=ps.sina, xv=xv, yv=yv, vx=vx, vy=vy)

    regrid_fixtures(args.ref)

    # 5. reference CPU FMM on random blobs (cross-check of the FMM path)
    x, y, g, sigma = rand_blobs(4096, 0.01, 17)
    vx, vy = ref.fmm_velocity(x, y, g, sigma, tol=1e-6)
    np.savez_compressed(os.path.join(HERE, "fmm_rand.npz"), x=x, y=y, g=g, sigma=sigma,
                        tol=1e-6, vx=vx, vy=vy)
    population_control_fixtures(args.ref)
    tutty_fixtures(args.ref)
    vorticity_fixtures()
    influence_fixtures()
    cutoff_fixtures()
    source_panel_fixtures()
    print("golden fixtures written to", HERE)


def m4_fixture():
    """0. the reference's own M4' weight loop on a sweep of points (the branch
    boundaries |x| = 0, 1, 2 exactly, points just inside and outside them,
    and a dense grid) for several Wee coefficients."""
    base = np.concatenate([np.linspace(-2.5, 2.5, 2001),
                           np.array([0.0, 1.0, -1.0, 2.0, -2.0]),
                           np.nextafter(np.array([1.0, 1.0, 2.0, 2.0]), np.array([0.0, 3.0, 0.0, 3.0])),
                           np.random.Generator(np.random.PCG64(5)).uniform(-2.2, 2.2, 3000)])
    cs = np.array([0.0, 0.1, 0.3, 0.7])
    w = np.stack([ref.m4kernel_1d(base, c) for c in cs])
    np.savez_compressed(os.path.join(HERE, "m4_ref.npz"), x=base, c=cs, w=w)


def regrid_fixtures(refroot):
    """4. remesh through the reference Regrid (with the reference's own M4'
    loop): C1 lattice, random blobs with and without the Wee diffusion term,
    and blobs sitting exactly on nodes."""
    m4_fixture()
    c1 = wl.lamb_oseen_lattice()
    R = load_reference_regrid(refroot)
    xb, yb = c1.bounds()
    xn, yn, gn = R.Regrid(c1.x, c1.y, c1.g, c1.sigma, c1.overlap, xb, yb, 0, 0.0)
    np.savez_compressed(os.path.join(HERE, "regrid_c1.npz"), x=c1.x, y=c1.y, g=c1.g,
                        sigma=c1.sigma, overlap=c1.overlap, xb=xb, yb=yb, c=0.0,
                        xn=xn, yn=yn, gn=gn)
    x, y, g, sigma = rand_blobs(2000, 0.01, 13, -0.3, 0.4)
    h = sigma * 0.8
    # blobs exactly on lattice nodes: |u| hits 0, 1 and 2 exactly
    x[:50] = (np.arange(50) - 20) * h + 0.5 * h + (-1.5 * h)
    y[:50] = 0.5 * h + (-1.5 * h)
    for tag, c in (("c0", 0.0), ("c3", 0.3)):
        xb = np.array([-1.5 * h, 1.5 * h])
        xn, yn, gn = R.Regrid(x, y, g, sigma, 0.8, xb, xb, 0, c)
        np.savez_compressed(os.path.join(HERE, f"regrid_rand_{tag}.npz"), x=x, y=y, g=g,
                            sigma=sigma, overlap=0.8, xb=xb, yb=xb, c=c, xn=xn, yn=yn, gn=gn)
    # a sparse set: the same blobs plus a few far from them (the dense lattice
    # window would hold ~1e11 cells)
    xf = np.concatenate([x, np.array([2000.0, 2000.0013, -1500.25, 3.0])])
    yf = np.concatenate([y, np.array([-0.2, -0.2021, 1800.5, -2500.0])])
    gf = np.concatenate([g, np.array([0.5, -0.25, 1.0, 2.0]) / 2000])
    xb = np.array([-1.5 * h, 1.5 * h])
    xn, yn, gn = R.Regrid(xf, yf, gf, sigma, 0.8, xb, xb, 0, 0.0)
    np.savez_compressed(os.path.join(HERE, "regrid_far.npz"), x=xf, y=yf, g=gf, sigma=sigma,
                        overlap=0.8, xb=xb, yb=xb, c=0.0, xn=xn, yn=yn, gn=gn)



def influence_fixtures():
    """9. the reference Cython assemble_influenceMatrix for 96 panels on the unit
    cylinder, collocation points at the panel centres moved slightly inside."""
    ps = wl.cylinder_panels(96, config=3, instance=11)
    xc = 0.5 * (ps.xs + ps.xe)
    yc = 0.5 * (ps.ys + ps.ye)
    nx, ny = ps.sina, -ps.cosa  # inward of a counter-clockwise contour
    r = np.hypot(xc, yc)
    s = -1.0 if np.mean(nx * xc / r + ny * yc / r) > 0 else 1.0
    xcp = xc + s * 1e-6 * nx
    ycp = yc + s * 1e-6 * ny
    A = ref.panel_influence(xcp, ycp, ps.xs, ps.ys, ps.xe, ps.ye, ps.cosa, ps.sina)
    np.savez_compressed(os.path.join(HERE, "panel_influence.npz"), xcp=xcp, ycp=ycp, xs=ps.xs,
                        ys=ps.ys, xe=ps.xe, ye=ps.ye, cosa=ps.cosa, sina=ps.sina, A=A)


def vorticity_fixtures():
    """8. the reference induced-vorticity loop: C1 lattice at the blobs, and
    random blobs (a duplicated blob, a zero one, a far one) at separate points."""
    c1 = wl.lamb_oseen_lattice()
    w = ref.vorticity_gauss(c1.x, c1.y, c1.g, c1.ksigmasqr)
    np.savez_compressed(os.path.join(HERE, "vort_c1.npz"), x=c1.x, y=c1.y, g=c1.g,
                        sigma=c1.sigma, ksigmasqr=c1.ksigmasqr, w=w)
    x, y, g, sigma = rand_blobs(3000, 0.01, 31)
    x[10], y[10] = x[11], y[11]
    g[20] = 0.0
    x[30], y[30] = 25.0, -13.0
    rng = np.random.Generator(np.random.PCG64(37))
    xt, yt = rng.uniform(-0.1, 1.1, 1500), rng.uniform(-0.1, 1.1, 1500)
    xt[:5], yt[:5] = x[:5], y[:5]
    k2 = 2.0 * sigma * sigma
    w = ref.vorticity_gauss(x, y, g, k2, xt, yt)
    np.savez_compressed(os.path.join(HERE, "vort_rand.npz"), x=x, y=y, g=g, sigma=sigma,
                        ksigmasqr=k2, xt=xt, yt=yt, w=w)


def cutoff_fixtures():
    """9. the reference's cutoff-kernel loops (vv2par_C_cpu.c, ww2par_C_cpu.c,
    extracted into oracle/_ref/): the C1 lattice at the blobs with sigmasqr =
    sigma^2, and random blobs (a duplicated blob, a zero one, a far one) at
    separate points, a few of them on blobs."""
    assert ref.cutoff_available(), "build oracle/_ref first: make -C oracle ref"
    c1 = wl.lamb_oseen_lattice()
    s2 = c1.sigma * c1.sigma
    vx, vy = ref.velocity_cutoff(c1.x, c1.y, c1.g, s2)
    w = ref.vorticity_cutoff(c1.x, c1.y, c1.g, s2)
    np.savez_compressed(os.path.join(HERE, "cutoff_c1.npz"), x=c1.x, y=c1.y, g=c1.g,
                        sigma=c1.sigma, sigmasqr=s2, vx=vx, vy=vy, w=w)
    x, y, g, sigma = rand_blobs(3000, 0.01, 41)
    x[10], y[10] = x[11], y[11]
    g[20] = 0.0
    x[30], y[30] = 25.0, -13.0
    rng = np.random.Generator(np.random.PCG64(43))
    xt, yt = rng.uniform(-0.1, 1.1, 1500), rng.uniform(-0.1, 1.1, 1500)
    xt[:5], yt[:5] = x[:5], y[:5]
    s2 = sigma * sigma
    vx, vy = ref.velocity_cutoff(x, y, g, s2, xt, yt)
    w = ref.vorticity_cutoff(x, y, g, s2, xt, yt)
    np.savez_compressed(os.path.join(HERE, "cutoff_rand.npz"), x=x, y=y, g=g, sigma=sigma,
                        sigmasqr=s2, xt=xt, yt=yt, vx=vx, vy=vy, w=w)


def source_panel_fixtures():
    """10. the reference's Cython constant-source panel kernel: velocity of
    64 panels on a circle (seeded strengths) at points around it (a few on
    panel 0's line extension and next to its midpoint), and the influence
    matrix on the collocation points (moved inside by a tenth of the panel
    length, as Panels places them)."""
    assert ref.source_panel_available(), "build oracle/_ref first: make -C oracle ref"
    ps = wl.cylinder_panels(64, instance=3)
    rng = np.random.Generator(np.random.PCG64(47))
    r = rng.uniform(1.0005, 3.0, 2000)
    t = rng.uniform(-np.pi, np.pi, 2000)
    xv, yv = r * np.cos(t), r * np.sin(t)
    dx, dy = ps.xe[0] - ps.xs[0], ps.ye[0] - ps.ys[0]
    xv[:3] = ps.xe[0] + dx * np.array([0.5, 1.0, 3.0])
    yv[:3] = ps.ye[0] + dy * np.array([0.5, 1.0, 3.0])
    xv[3] = 0.5 * (ps.xs[0] + ps.xe[0]) - 1e-6 * dy
    yv[3] = 0.5 * (ps.ys[0] + ps.ye[0]) + 1e-6 * dx
    vx, vy = ref.source_panel_velocity(ps.gamma, ps.xs, ps.ys, ps.xe, ps.ye, ps.cosa, ps.sina,
                                       xv, yv)
    L = np.sqrt((ps.xe - ps.xs) ** 2 + (ps.ye - ps.ys) ** 2)
    xcp = 0.5 * (ps.xs + ps.xe) + ps.sina * L * 0.1
    ycp = 0.5 * (ps.ys + ps.ye) - ps.cosa * L * 0.1
    A = ref.source_panel_influence(xcp, ycp, ps.xs, ps.ys, ps.xe, ps.ye, ps.cosa, ps.sina)
    np.savez_compressed(os.path.join(HERE, "source_panel.npz"), sigma=ps.gamma, xs=ps.xs,
                        ys=ps.ys, xe=ps.xe, ye=ps.ye, cosa=ps.cosa, sina=ps.sina, xv=xv, yv=yv,
                        vx=vx, vy=vy, xcp=xcp, ycp=ycp, A=A)


def tutty_fixtures(refroot):
    """7. the reference diffusion_tutty on random blobs (with blobs exactly on
    lattice nodes) for hNu/h = 0.5 and for hNu = 0, and on the C1 lattice."""
    tutty = load_reference_tutty(refroot)
    x, y, g, sigma = rand_blobs(2000, 0.01, 29, -0.3, 0.4)
    h = sigma * 0.8
    x[:40] = (np.arange(40) - 20) * h + 0.5 * h + (-1.5 * h)
    y[:40] = 0.5 * h + (-1.5 * h)
    xb = np.array([-1.5 * h, 1.5 * h])
    cases = [("rand", x, y, g, sigma, 0.8, xb, 0.25 * h * h, 1.0),
             ("rand_nu0", x, y, g, sigma, 0.8, xb, 0.01, 0.0)]
    c1 = wl.lamb_oseen_lattice()
    c1b, _ = c1.bounds()
    cases.append(("c1", c1.x, c1.y, c1.g, c1.sigma, c1.overlap, c1b, 1e-4, 0.5))
    for tag, xa, ya, ga, sg, ov, bnd, dt, nu in cases:
        xn, yn, gn = tutty(dt, nu, sg * ov, xa.copy(), ya.copy(), ga.copy(), sg, bnd, bnd,
                           overlap=ov)
        np.savez_compressed(os.path.join(HERE, f"tutty_{tag}.npz"), x=xa, y=ya, g=ga, sigma=sg,
                            overlap=ov, xb=bnd, yb=bnd, dt=dt, nu=nu, xn=xn, yn=yn, gn=gn)


def population_control_fixtures(refroot):
    """6. the reference PopulationControl on (a) the C1 remesh output (explicit
    zeros, default thresholds), (b) circulations spread over 12 decades with a
    threshold that must drop several decades, (c) a global limit 30 decades
    below the local threshold (more than 16 decade steps), with exact zeros and
    ties at the thresholds."""
    R = load_reference_regrid(refroot)
    c1 = wl.lamb_oseen_lattice()
    xb, yb = c1.bounds()
    xn, yn, gn = R.Regrid(c1.x, c1.y, c1.g, c1.sigma, c1.overlap, xb, yb, 0, 0.0)
    cases = [("c1", xn, yn, gn, 1e-8, 1e-8)]
    rng = np.random.Generator(np.random.PCG64(23))
    n = 5000
    x = rng.uniform(-1, 1, n)
    y = rng.uniform(-1, 1, n)
    g = np.sign(rng.standard_normal(n)) * 10.0 ** rng.uniform(-14, -2, n)
    g[:5] = 0.0
    g[5:10] = 1e-3  # exactly at the starting threshold: kept (|g| < thr is false)
    cases.append(("decades", x, y, g, 1e-3, 1e-6))
    g2 = np.sign(rng.standard_normal(n)) * 10.0 ** rng.uniform(-45, -1, n)
    g2[:3] = 0.0
    cases.append(("deep", x, y, g2, 1.0, 1e-30))
    for tag, xa, ya, ga, tl, tg in cases:
        xo, yo, go = R.PopulationControl(xa.copy(), ya.copy(), ga.copy(), tl, tg)
        np.savez_compressed(os.path.join(HERE, f"popctl_{tag}.npz"), x=xa, y=ya, g=ga,
                            thr_local=tl, thr_global=tg, xo=xo, yo=yo, go=go)


if __name__ == "__main__":
    main()
