"""Synthetic workloads of the IPM hot path, as reference-schema TOML configs.

Each workload is a UQCreator input file (sections [general] [mesh] [problem]
[moment_system], read exactly as code/src/settings.cpp:22-323 reads them) plus
a [uqc] table that the reference ignores and this package reads:

  ic          initial-state parameters of the problem (see below)
  bounds      bounded-barrier ansatz bounds (u_minus, u_plus)
  mesh        "uniform1d" (the reference's Mesh1D) or "tri_jitter" (seeded
              jittered triangle mesh on [0,1]^2, nx x ny rectangles x 2)
  mesh_params [nx, ny, jitter, seed] for tri_jitter
  precision   "fp64" (plain form) or "mixed" (tensor-core Hessian)
  newton      "reference", "guarded" or "safe" Newton (see euler2d)
  steps       stop after this many time steps (0: run to tEnd only)
  refinementIndicator   "moments" (the code's sum of |u(0, i)|, default) or
              "energy" (the paper's S_l) for the level rule
  refinementBounds      [lower, upper] of the level rule (default [0.004, 0.02])
  retardationLevels / retardationResiduals   the highest refinement level
              allowed, raised to retardationLevels[k] once the residual has
              fallen below retardationResiduals[k-1] (one fewer residuals)

Problems and their ic parameters:
  Burgers1D       [uL, uR, x0, x1]          ramp of code/src/burgers.cpp:48-68
  Euler1D         [] or [x0, rhoL, pL, rhoR, pR]   the reference's fixed Sod state (euler.cpp:95-128)
  Euler2D         [xs, rhoL, pL, rhoR, pR]  Sod-type interface at x = xs + s0 xi0
  ShallowWater1D  [xd, hL, hR]              dam break h = hL (1 + s0 xi0) | hR
"""
from __future__ import annotations

import tomllib

_TEMPLATE = """[general]
problem = "{problem}"
outputDir = "out"
writeFrequency = 100000000

[mesh]
dimension = {dim}
numberOfCells = {ncells}
a = {a}
b = {b}
outputFile = "{name}"
{mesh_extra}
[problem]
timestepping = "explicitEuler"
distribution = [[{dists}],[{sigmas}]]
CFL = {cfl}
tEnd = {tend}
{extra_problem}
[moment_system]
closure = "{closure}"
moments = [["{degtype}"],[{degrees}]]
quadPoints = [["tensorizedGrid"],[{quads}]]
maxIterations = {maxit}
epsilon = {eps}

[uqc]
ic = [{ic}]
bounds = [{bounds}]
mesh = "{mesh}"
mesh_params = [{mesh_params}]
precision = "{precision}"
newton = "{newton}"
steps = {steps}
{uqc_extra}"""


def make_toml(*, name, problem, closure, dim, ncells=0, a=0.0, b=1.0, sigmas, cfl, tend, degrees,
              nquad, ic, bounds=(3.0, 12.0), mesh="uniform1d", mesh_params=(0, 0, 0.0, 0),
              maxit=1000, eps=1e-10, degtype="totalDegree", precision="fp64", gamma=None,
              newton="reference", steps=0, mesh_extra="", uqc_extra="") -> str:
    degrees = list(degrees)
    quads = [nquad] * len(degrees)
    extra = f"gamma = {gamma!r}\n" if gamma is not None else ""
    return _TEMPLATE.format(
        name=name, problem=problem, closure=closure, dim=dim, ncells=ncells, a=float(a), b=float(b),
        dists=",".join('"Legendre"' for _ in sigmas), sigmas=",".join(repr(float(s)) for s in sigmas),
        cfl=repr(float(cfl)), tend=repr(float(tend)), extra_problem=extra, degtype=degtype,
        degrees=",".join(str(int(d)) for d in degrees), quads=",".join(str(int(q)) for q in quads),
        maxit=int(maxit), eps=repr(float(eps)), ic=",".join(repr(float(v)) for v in ic),
        bounds=",".join(repr(float(v)) for v in bounds), mesh=mesh,
        mesh_params=",".join(repr(v) if isinstance(v, float) else str(v) for v in mesh_params),
        precision=precision, newton=newton, steps=int(steps), mesh_extra=mesh_extra, uqc_extra=uqc_extra)


def burgers1d(ncells=500, tend=0.11, degree=4, nquad=20, eps=1e-10, x0=0.5, **kw) -> str:
    """Plain IPM FP64 Burgers: x in [0,3], u=12 left of x0+0.2 xi (x0 = 0.5), ramp of
    width 0.1 down to 3, bounded barrier (2.5, 12.5), local Lax-Friedrichs flux, CFL 0.5."""
    return make_toml(name="burgers1d", problem="Burgers1D", closure="BoundedBarrier", dim=1, ncells=ncells,
                     a=0.0, b=3.0, sigmas=[0.2], cfl=0.5, tend=tend, degrees=[degree], nquad=nquad,
                     ic=[12.0, 3.0, x0, x0 + 0.1], bounds=(2.5, 12.5), eps=eps, **kw)


def euler2d(nx=400, ny=250, degree=5, nquad=10, dim_xi=2, tend=0.2, cfl=0.5, eps=1e-10, seed=7,
            jitter=0.2, newton="guarded", xs=0.5, **kw) -> str:
    """2-D Euler (gamma 1.4) on a jittered triangle mesh of nx*ny*2 cells, Sod-type
    interface x = 0.5 + 0.05 xi1, left density 1 + 0.1 xi2 (and left pressure
    1 + 0.1 xi3 when dim_xi = 3), right state (0.125, 0.1), total-degree basis.

    Newton runs "guarded": the reference's SolveClosure accepts a trial step
    whose residual norm is NaN (code/src/closure.cpp:172) and then fails in posv
    for cells inside the uncertain interface band; the guard rejects such steps
    as SolveClosureSafe does (closure.cpp:318)."""
    sig = [0.05, 0.1, 0.1][:dim_xi]
    return make_toml(name="euler2d", problem="Euler2D", closure="Euler2D", dim=2, ncells=nx * ny * 2,
                     sigmas=sig, cfl=cfl, tend=tend, degrees=[degree], nquad=nquad,
                     ic=[xs, 1.0, 1.0, 0.125, 0.1], mesh="tri_jitter", mesh_params=(nx, ny, float(jitter), seed),
                     eps=eps, gamma=1.4, newton=newton, **kw)


def shallow_water1d(ncells=1_000_000, max_degree=9, nquad=30, tend=0.05, eps=1e-10, **kw) -> str:
    """1-D shallow water dam break h_L = 1 + 0.2 xi, h_R = 0.5 on [0,1], adaptive
    per-cell degree 1..max_degree (levels of the reference's refinement scheme)."""
    return make_toml(name="sw1d", problem="ShallowWater1D", closure="ShallowWater", dim=1, ncells=ncells,
                     a=0.0, b=1.0, sigmas=[0.2], cfl=0.5, tend=tend, degrees=list(range(1, max_degree + 1)),
                     nquad=nquad, ic=[0.5, 1.0, 0.5], eps=eps, **kw)


def euler1d(ncells=400, degree=4, nquad=10, tend=0.1, cfl=0.5, eps=1e-10, sigma=0.05, newton="guarded", sigmas=None,
            **kw) -> str:
    """1-D Euler (gamma 1.4) on [0, 1]: the reference's own Sod state (euler.cpp:95-128,
    interface x = 0.3 + sigma xi, left (1, 0, 1), right density and pressure 0.3),
    EulerClosure (three states), HLL flux."""
    return make_toml(name="euler1d", problem="Euler1D", closure="Euler", dim=1, ncells=ncells, a=0.0, b=1.0,
                     sigmas=sigmas or [sigma], cfl=cfl, tend=tend, degrees=[degree], nquad=nquad, ic=[], eps=eps, gamma=1.4,
                     newton=newton, **kw)


def euler2d_3u(nx=512, ny=256, degree=4, nquad=8, **kw) -> str:
    """Large 2-D Euler with 3 uncertainties, total degree 4 (35 moments x 4 states), 8^3 nodes."""
    return euler2d(nx=nx, ny=ny, degree=degree, nquad=nquad, dim_xi=3, **kw)


def serving_stream(n_requests=2000, rate_per_s=50.0, seed=11, steps=(5, 40), euler_fraction=0.5, scale=1.0):
    """Seeded request stream of the serving workload: Poisson arrivals (rate
    rate_per_s) of UQ solves mixing 1-D Burgers (200-20k cells, degree 2-9:
    3-10 moments) and 2-D Euler (10k-200k cells, total degree 2-5: 6-21
    moments, 2 uncertainties), each with its shock / interface offset drawn from
    U[0.05, 0.3] and a horizon of `steps` time steps (drawn uniformly, the
    [uqc] steps limit; tEnd is far beyond). scale < 1 shrinks the meshes.
    Returns [(arrival_s, kind, toml)]."""
    import numpy as np
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for _ in range(n_requests):
        t += rng.exponential(1.0 / rate_per_s)
        off = float(rng.uniform(0.05, 0.3))
        nsteps = int(rng.integers(steps[0], steps[1] + 1))
        if rng.random() < euler_fraction:
            cells = int(rng.integers(10_000, 200_001) * scale)
            deg = int(rng.integers(2, 6))
            nx = max(4, int(round((cells / 2 * 1.6) ** 0.5)))
            ny = max(2, cells // (2 * nx))
            toml = euler2d(nx=nx, ny=ny, degree=deg, nquad=2 * deg, tend=10.0, xs=0.5 - off, steps=nsteps)
            out.append((t, "euler2d", toml))
        else:
            cells = max(20, int(rng.integers(200, 20_001) * scale))
            deg = int(rng.integers(2, 10))
            toml = burgers1d(ncells=cells, degree=deg, nquad=4 * deg + 4, tend=10.0, x0=0.5 + off, steps=nsteps)
            out.append((t, "burgers1d", toml))
    return out


WORKLOADS = {
    "burgers1d": burgers1d,
    "euler2d": euler2d,
    "sw1d": shallow_water1d,
    "euler2d_3u": euler2d_3u,
    "euler1d": euler1d,
}


def parse(toml_text: str) -> dict:
    return tomllib.loads(toml_text)


# --------------------------------------------------------------------------
# Seeded jittered triangle mesh ("tri_jitter"). The C++ host builds the same
# mesh (csrc/host/mesh.cpp); a CPU test checks that both agree bit for bit.

_M64 = (1 << 64) - 1


def _splitmix64(x):
    import numpy as np
    x = np.asarray(x, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = x + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def tri_jitter_mesh(nx: int, ny: int, jitter: float = 0.2, seed: int = 7) -> dict:
    """Nodes (i, j) at ((i + a r_x) / nx, (j + a r_y) / ny) with r uniform in [-1, 1)
    from SplitMix64(seed * 2^32 + 2 node + c) for interior nodes (a = jitter) and
    exact grid positions on the boundary. Rectangle (i, j) splits along a-c into
    (a, b, c), (a, c, d); the two corner rectangles whose corner node is b or d
    split along b-d into (a, b, d), (b, c, d) so no triangle has three boundary
    nodes. Cell id = 2 (j nx + i) + t."""
    import numpy as np
    nn = (nx + 1) * (ny + 1)
    node = np.arange(nn, dtype=np.int64)
    i = node % (nx + 1)
    j = node // (nx + 1)
    bnd = ((i == 0) | (i == nx) | (j == 0) | (j == ny)).astype(np.int32)
    key = np.uint64(seed) * np.uint64(1 << 32) + np.uint64(2) * node.astype(np.uint64)
    rx = (_splitmix64(key) >> np.uint64(11)).astype(np.float64) * 2.0 ** -53
    ry = (_splitmix64(key + np.uint64(1)) >> np.uint64(11)).astype(np.float64) * 2.0 ** -53
    fx = i.astype(np.float64)
    fy = j.astype(np.float64)
    x = np.where(bnd == 1, fx / nx, (fx + jitter * (2.0 * rx - 1.0)) / nx)
    y = np.where(bnd == 1, fy / ny, (fy + jitter * (2.0 * ry - 1.0)) / ny)
    xy = np.stack([x, y], axis=1)
    ri = np.arange(nx * ny, dtype=np.int64)
    ii = ri % nx
    jj = ri // nx
    a = jj * (nx + 1) + ii
    b = a + 1
    c = a + nx + 2
    d = a + nx + 1
    flip = ((ii == 0) & (jj == ny - 1)) | ((ii == nx - 1) & (jj == 0))
    t0 = np.where(flip[:, None], np.stack([a, b, d], 1), np.stack([a, b, c], 1))
    t1 = np.where(flip[:, None], np.stack([b, c, d], 1), np.stack([a, c, d], 1))
    tri = np.stack([t0, t1], axis=1).reshape(-1, 3).astype(np.int32)
    return dict(xy=xy, node_boundary=bnd, tri=tri)


def su2_channel(nx: int, ny: int, jitter: float = 0.2, seed: int = 7, slant: float = 0.25, shuffle: int = 5) -> str:
    """SU2 text (the format Mesh2D::LoadSU2MeshFromFile reads, mesh2d.cpp:68-259)
    of the tri_jitter mesh mapped to a channel whose right wall leans,
    x' = x (1 + slant y). Markers "inlet" (x = 0), "outlet" (the leaning
    wall), "bottom", "top" as line elements "3 a b". Node lines carry their
    ids in a seeded shuffled order (the reader sorts them)."""
    import numpy as np
    m = tri_jitter_mesh(nx, ny, jitter, seed)
    xy = m["xy"].copy()
    xy[:, 0] = xy[:, 0] * (1.0 + slant * xy[:, 1])
    tri = m["tri"]
    node = lambda i, j: j * (nx + 1) + i
    out = ["% channel with a leaning right wall", "NDIME= 2", f"NELEM= {len(tri)}"]
    out += [f"5 {a} {b} {c} {e}" for e, (a, b, c) in enumerate(tri)]
    order = np.random.default_rng(shuffle).permutation(len(xy)) if shuffle else np.arange(len(xy))
    out.append(f"NPOIN= {len(xy)}")
    out += [f"{float(xy[n, 0])!r} {float(xy[n, 1])!r} {n}" for n in order]
    markers = {
        "inlet": [(node(0, j), node(0, j + 1)) for j in range(ny)],
        "outlet": [(node(nx, j), node(nx, j + 1)) for j in range(ny)],
        "bottom": [(node(i, 0), node(i + 1, 0)) for i in range(nx)],
        "top": [(node(i, ny), node(i + 1, ny)) for i in range(nx)],
    }
    out.append(f"NMARK= {len(markers)}")
    for tag, elems in markers.items():
        out += [f"MARKER_TAG= {tag}", f"MARKER_ELEMS= {len(elems)}"]
        out += [f"3 {a} {b}" for a, b in elems]
    return "\n".join(out) + "\n"


def euler2d_su2(mesh_file: str, bcs=(("inlet", "dirichlet"), ("outlet", "noslip"), ("bottom", "swwall"), ("top", "swwall")),
                degree=5, nquad=10, dim_xi=2, tend=0.2, cfl=0.5, eps=1e-10, newton="guarded", xs=0.7, **kw) -> str:
    """2-D Euler (the euler2d problem) on an SU2 mesh: [mesh] format = "SU2",
    SU2MeshFile (relative to the config's directory) and SU2BC markers
    (mesh2d.cpp:21-56). Walls reflect the flow through ghost states
    (expliciteuler.cpp:24-70)."""
    sig = [0.05, 0.1, 0.1][:dim_xi]
    bc = ", ".join(f'["{t}", "{k}"]' for t, k in bcs)
    extra = f'format = "SU2"\nSU2MeshFile = "{mesh_file}"\nSU2BC = [{bc}]\n'
    return make_toml(name="euler2d_su2", problem="Euler2D", closure="Euler2D", dim=2, ncells=0, sigmas=sig, cfl=cfl,
                     tend=tend, degrees=[degree], nquad=nquad, ic=[xs, 1.0, 1.0, 0.125, 0.1], eps=eps, gamma=1.4,
                     newton=newton, mesh_extra=extra, **kw)


def mesh_for(toml_text: str):
    """The 2-D mesh arrays a config describes, or None for 1-D configs."""
    d = parse(toml_text)
    u = d.get("uqc", {})
    if u.get("mesh", "uniform1d") != "tri_jitter":
        return None
    nx, ny, jit, seed = u["mesh_params"]
    return tri_jitter_mesh(int(nx), int(ny), float(jit), int(seed))
