"""Closed triangle meshes for the mesh-seeding tests (layout of TriangleMesh: vertices (V,3) float64, triangles
(T,4) int64 = three vertex ids and a normal id)."""
import numpy as np


def box(lo, hi):
    lo, hi = np.asarray(lo, float), np.asarray(hi, float)
    V = np.array([[lo[0] if (c & 1) == 0 else hi[0], lo[1] if (c & 2) == 0 else hi[1], lo[2] if (c & 4) == 0 else hi[2]]
                  for c in range(8)])
    quads = [(0, 2, 3, 1), (4, 5, 7, 6), (0, 1, 5, 4), (2, 6, 7, 3), (0, 4, 6, 2), (1, 3, 7, 5)]
    T = []
    for a, b, c, d in quads:
        T += [(a, b, c, 0), (a, c, d, 0)]
    return V, np.array(T, dtype=np.int64)


def icosphere(center, radius, subdiv=2):
    t = (1.0 + 5 ** 0.5) / 2.0
    V = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    F = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
         (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7),
         (9, 8, 1)]
    V = [np.array(v, float) / np.linalg.norm(v) for v in V]
    for _ in range(subdiv):
        cache, F2 = {}, []

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = V[a] + V[b]
                V.append(m / np.linalg.norm(m))
                cache[key] = len(V) - 1
            return cache[key]

        for a, b, c in F:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            F2 += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        F = F2
    V = np.array(V) * radius + np.asarray(center, float)
    T = np.array([(a, b, c, 0) for a, b, c in F], dtype=np.int64)
    return V, T


def write_obj(path, V, T, name="mesh", N=None):
    """A mesh as OBJ text that OBJManager::Load reads ("v" and "vn" lines, "f a//n b//n c//n" faces with 1-based ids;
    with normals N, each face's normal is N[T[:, 3]], else one normal (0, 0, 1) for all)."""
    lines = [f"o {name}"] + [f"v {x:.17g} {y:.17g} {z:.17g}" for x, y, z in V]
    if N is None:
        lines += ["vn 0 0 1"]
        lines += [f"f {a + 1}//1 {b + 1}//1 {c + 1}//1" for a, b, c, *_ in T]
    else:
        lines += [f"vn {x:.17g} {y:.17g} {z:.17g}" for x, y, z in N]
        lines += [f"f {a + 1}//{n + 1} {b + 1}//{n + 1} {c + 1}//{n + 1}" for a, b, c, n in T]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def with_face_normals(V, T):
    """(V, T, N): each triangle's normal id set to its own index into N, the unit face normals (b - a) x (c - a)."""
    V = np.asarray(V, float)
    T = np.array(T, dtype=np.int64)
    a, b, c = V[T[:, 0]], V[T[:, 1]], V[T[:, 2]]
    N = np.cross(b - a, c - a)
    N /= np.linalg.norm(N, axis=1, keepdims=True)
    T[:, 3] = np.arange(T.shape[0])
    return V, T, N
