"""Writes the mesh and image assets the .luz test scenes in this folder load:
octahedron.obj (unit octahedron with vertex normals and texture coordinates),
checker_cross.ppm (12x9 checker in a 4x3 cube-cross atlas) and sky_small.ppm
(16x8 equirect sky). Run from this folder; the outputs are committed."""
import math


def octahedron(path):
    v = [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]
    faces = [(0, 2, 4), (4, 2, 1), (1, 2, 5), (5, 2, 0), (4, 3, 0), (1, 3, 4), (5, 3, 1), (0, 3, 5)]
    with open(path, "w") as f:
        f.write("# octahedron, unit radius\n")
        for p in v:
            f.write("v %g %g %g\n" % p)
        for p in v:
            f.write("vn %g %g %g\n" % p)
        for p in v:
            f.write("vt %.6f %.6f\n" % (0.5 + math.atan2(p[2], p[0]) / (2 * math.pi), 0.5 + p[1] * 0.5))
        for a, b, c in faces:
            f.write("f %d/%d/%d %d/%d/%d %d/%d/%d\n" % (a + 1, a + 1, a + 1, b + 1, b + 1, b + 1, c + 1, c + 1, c + 1))


def ppm(path, w, h, fn):
    with open(path, "w") as f:
        f.write("P3\n%d %d\n255\n" % (w, h))
        for y in range(h):
            f.write(" ".join("%d %d %d" % fn(x, y) for x in range(w)) + "\n")


if __name__ == "__main__":
    octahedron("octahedron.obj")
    ppm("checker_cross.ppm", 12, 9, lambda x, y: (230, 70, 40) if (x // 3 + y // 3) % 2 == 0
        else ((40, 90, 220) if (x + y) % 2 else (250, 240, 200)))
    ppm("sky_small.ppm", 16, 8, lambda x, y: (min(255, 60 + y * 20), min(255, 90 + y * 18), 255 if y < 4 else 180 - y * 10))
