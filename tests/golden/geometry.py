"""Seeded synthetic geometries of the benchmark workloads (Angstrom).

* water cluster: rigid monomers (O-H 0.9572 A, H-O-H 104.52 deg) with O on the
  sites of a cubic lattice (3.0 A spacing), each monomer turned by a uniform
  random rotation (Shoemake's quaternion method, K. Shoemake, "Uniform random
  rotations", Graphics Gems III, 1992) and shifted by a uniform jitter of
  +-a A per Cartesian component; all draws from numpy.random.default_rng(seed)
  in lattice order.
* all-trans linear alkane CnH2n+2: planar zig-zag backbone (C-C 1.54 A,
  C-C-C 109.4712 deg), C-H 1.09 A, tetrahedral hydrogens.

These generate the inputs of the (H2O)_8, (H2O)_16, (H2O)_64 and C20H42
workloads; the fixtures under tests/golden carry the resulting atm/bas/env.
"""
import numpy

OH = 0.9572
HOH = numpy.deg2rad(104.52)
SPACING = 3.0


def water_monomer():
    h = 0.5 * HOH
    return [('O', numpy.zeros(3)),
            ('H', numpy.array([OH * numpy.sin(h), 0.0, OH * numpy.cos(h)])),
            ('H', numpy.array([-OH * numpy.sin(h), 0.0, OH * numpy.cos(h)]))]


def random_rotation(rng):
    u1, u2, u3 = rng.uniform(0.0, 1.0, 3)
    q = numpy.array([numpy.sqrt(1 - u1) * numpy.sin(2 * numpy.pi * u2),
                     numpy.sqrt(1 - u1) * numpy.cos(2 * numpy.pi * u2),
                     numpy.sqrt(u1) * numpy.sin(2 * numpy.pi * u3),
                     numpy.sqrt(u1) * numpy.cos(2 * numpy.pi * u3)])
    x, y, z, w = q
    return numpy.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def water_cluster(shape, jitter, seed, sites=None):
    """Water cluster on a cubic lattice of `shape` (nx, ny, nz); `sites`
    optionally restricts to a subset of lattice sites (list of index tuples)."""
    rng = numpy.random.default_rng(seed)
    if sites is None:
        sites = [(i, j, k) for i in range(shape[0]) for j in range(shape[1]) for k in range(shape[2])]
    atoms = []
    for s in sites:
        R = random_rotation(rng)
        shift = rng.uniform(-jitter, jitter, 3)
        origin = numpy.array(s, dtype=float) * SPACING + shift
        for sym, r in water_monomer():
            atoms.append((sym, origin + R @ r))
    return atoms


def alkane(n):
    cc, ch = 1.54, 1.09
    theta = numpy.deg2rad(109.4712)
    dx, dy = cc * numpy.sin(theta / 2), cc * numpy.cos(theta / 2)
    carbons = [numpy.array([i * dx, (i % 2) * dy, 0.0]) for i in range(n)]
    z = numpy.array([0.0, 0.0, 1.0])
    atoms = [('C', c) for c in carbons]
    cos_t = numpy.cos(theta)
    for i, c in enumerate(carbons):
        nbrs = [carbons[j] for j in (i - 1, i + 1) if 0 <= j < n]
        if len(nbrs) == 2:
            u = sum((m - c) / numpy.linalg.norm(m - c) for m in nbrs)
            b = -u / numpy.linalg.norm(u)
            half = 0.5 * theta
            for s in (1, -1):
                atoms.append(('H', c + ch * (numpy.cos(half) * b + s * numpy.sin(half) * z)))
        else:
            a = (c - nbrs[0]) / numpy.linalg.norm(c - nbrs[0])
            p = numpy.cross(z, a)
            p /= numpy.linalg.norm(p)
            if i == 0:
                p = -p
            # angle (C->H, C->neighbour) = theta: C->H = -cos(theta) a + sin(theta) e
            for phi in (0.0, 2 * numpy.pi / 3, 4 * numpy.pi / 3):
                e = numpy.cos(phi) * p + numpy.sin(phi) * z
                atoms.append(('H', c + ch * (-cos_t * a + numpy.sin(theta) * e)))
    return atoms


def workloads():
    """name -> (atoms, basis) for every workload the fixtures and the bench use."""
    return {
        'h2o_631g': ([('O', numpy.zeros(3)), ('H', numpy.array([0., -0.757, 0.587])),
                      ('H', numpy.array([0., 0.757, 0.587]))], '631g'),
        'h2o_vdz': ([('O', numpy.zeros(3)), ('H', numpy.array([0., -0.757, 0.587])),
                     ('H', numpy.array([0., 0.757, 0.587]))], 'cc-pvdz'),
        'h2o2_vtz': (water_cluster((2, 1, 1), 0.2, 202), 'cc-pvtz'),
        'h2o8_vdz': (water_cluster((2, 2, 2), 0.2, 101), 'cc-pvdz'),
        'c20h42_vdz': (alkane(20), 'cc-pvdz'),
        'h2o16_vdz': (water_cluster((2, 2, 4), 0.2, 505), 'cc-pvdz'),
        'h2o64_vtz': (water_cluster((4, 4, 4), 0.3, 303), 'cc-pvtz'),
        # the first 4 / 8 / 16 waters of the (H2O)64 geometry: bounded samples of
        # that workload for the CPU baseline and for scaling estimates
        'h2o64_vtz_sub4': (water_cluster((4, 4, 4), 0.3, 303)[:12], 'cc-pvtz'),
        'h2o64_vtz_sub8': (water_cluster((4, 4, 4), 0.3, 303)[:24], 'cc-pvtz'),
        'h2o64_vtz_sub16': (water_cluster((4, 4, 4), 0.3, 303)[:48], 'cc-pvtz'),
        # half of it: matrices above the 126 MB L2, the case profiled under ncu
        'h2o64_vtz_sub32': (water_cluster((4, 4, 4), 0.3, 303)[:96], 'cc-pvtz'),
    }
