"""Seeded synthetic scenes of the benchmark configurations.

  cornell_box()         plain small: procedural Cornell box, 36 f32 triangles, red/green/white diffuse
                        walls, 0.5 x 0.5 ceiling light (emission 15), rough-metal tall box (roughness 0.3),
                        glass short box (IOR 1.5), four solid 64 x 64 RGBA8 diffuse layers.
  icosphere_field()     plain at scale: 64 instances of seeded displaced icospheres (subdivision 5,
                        20,480 triangles each, 1.31M triangles) with random rigid transforms in a 20-unit
                        cube; roughness U[0.05, 1], 10% glass with IOR U[1.3, 1.7], 2% emissive with
                        log-normal(1, 1) brightness; 16-layer 1024 x 1024 value-noise textures.
  occluded_cornell()    indirect-heavy: the Cornell box lit by one 0.2 x 0.2 emitter behind an occluder.
  box_field(n_tris)     batched requests: Cornell-style scenes with n_tris triangles of subdivided boxes.

Cameras follow cgmath's perspective / look_to_rh conventions (examples/cornell_box/src/main.rs:500-507).
Material records and cameras are packed by a packer: by default the library's Material::new and
Camera::from_proj_view (LibraryPacker); any object with the same two methods can stand in for it, so
that a scene can be generated without loading the library at all.
"""
import math

import numpy as np

from .api import Camera, EmissionScale, Material, MaterialType


class Scene:
    def __init__(self):
        self.blas = []          # dicts: vertices (V, 3|4) f32, indices (T*3,) u32 or None, flags
        self.instances = []     # dicts: transform (12,), blas, material_indices (T,), mask
        self.materials = []
        self.diffuse, self.emission, self.attributes = [], [], []
        self.recolour = None
        self.sky = None         # (6, S, S, 4) u8 or None
        self.camera = None
        self.width, self.height = 256, 256
        self.name = ""

    @property
    def triangle_count(self):
        return sum((b["indices"].size // 3) if b.get("indices") is not None else b["vertices"].shape[0] // 3
                   for b in self.blas)

    def layout_counts(self):
        return (max(1, len(self.instances)), max(1, len(self.diffuse)), max(1, len(self.emission)),
                max(1, len(self.attributes)))


class LibraryPacker:
    """Packs through the library: Material::new (src/lib.rs:132-163) and Camera::from_proj_view
    (src/camera.rs:15-24)."""

    @staticmethod
    def material(uv1, uv2, uv3, recolour, diffuse, emission, attributes, emission_scale, ior, ty):
        return Material.new(uv1, uv2, uv3, recolour, diffuse, emission, attributes, emission_scale, ior, ty)

    @staticmethod
    def camera(proj, view):
        return Camera.new(proj, view)


def _packer(packer):
    return LibraryPacker if packer is None else packer


IDENTITY = np.array([1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0], dtype=np.float32)


# ---------------------------------------------------------------- cameras (cgmath semantics, column-major)
def perspective(fovy_deg, aspect, near, far):
    f = 1.0 / math.tan(math.radians(fovy_deg) / 2.0)
    m = np.zeros((4, 4), dtype=np.float64)  # m[col][row]
    m[0][0] = f / aspect
    m[1][1] = f
    m[2][2] = (far + near) / (near - far)
    m[2][3] = -1.0
    m[3][2] = (2.0 * far * near) / (near - far)
    return m.astype(np.float32)


def look_to_rh(eye, direction, up):
    f = np.asarray(direction, np.float64)
    f = f / np.linalg.norm(f)
    s = np.cross(f, up)
    s = s / np.linalg.norm(s)
    u = np.cross(s, f)
    e = np.asarray(eye, np.float64)
    m = np.zeros((4, 4), dtype=np.float64)
    m[0] = [s[0], u[0], -f[0], 0.0]
    m[1] = [s[1], u[1], -f[1], 0.0]
    m[2] = [s[2], u[2], -f[2], 0.0]
    m[3] = [-e.dot(s), -e.dot(u), e.dot(f), 1.0]
    return m.astype(np.float32)


def make_camera(eye, target, fovy_deg, aspect, up=(0.0, 1.0, 0.0), packer=None):
    d = np.asarray(target, np.float64) - np.asarray(eye, np.float64)
    return _packer(packer).camera(perspective(fovy_deg, aspect, 0.1, 200.0),
                                  look_to_rh(eye, d, np.asarray(up, np.float64)))


def solid(rgba, size=64):
    return np.tile(np.asarray(rgba, np.uint8).reshape(1, 1, 4), (size, size, 1))


UV = ((1.0, 1.0), (0.0, 1.0), (1.0, 0.0))


def _mat(diffuse, emission=None, attributes=None, scale=1.0, ior=None, ty=MaterialType.Diffuse, uv=UV, packer=None):
    return _packer(packer).material(uv[0], uv[1], uv[2], (0, 0), diffuse, emission, attributes,
                                    EmissionScale.from_emission_scale(scale), ior, ty)


def _quad(p0, p1, p2, p3):
    """Two triangles (p0, p1, p2), (p0, p2, p3); counter-clockwise seen from the normal side."""
    return [p0, p1, p2, p0, p2, p3]


def _box(center, size, angle_deg):
    """12 triangles of an axis box rotated about +y, wound counter-clockwise seen from outside."""
    cx, cy, cz = center
    sx, sy, sz = size
    a = math.radians(angle_deg)
    ca, sa = math.cos(a), math.sin(a)

    def P(x, y, z):
        x, z = x * sx / 2, z * sz / 2
        return (cx + ca * x + sa * z, cy + y * sy, cz - sa * x + ca * z)

    c = {k: P(*k) for k in [(x, y, z) for x in (-1, 1) for y in (0, 1) for z in (-1, 1)]}
    tris = []
    tris += _quad(c[(-1, 1, -1)], c[(-1, 1, 1)], c[(1, 1, 1)], c[(1, 1, -1)])      # top (+y)
    tris += _quad(c[(-1, 0, -1)], c[(1, 0, -1)], c[(1, 0, 1)], c[(-1, 0, 1)])      # bottom (-y)
    tris += _quad(c[(-1, 0, 1)], c[(1, 0, 1)], c[(1, 1, 1)], c[(-1, 1, 1)])        # +z
    tris += _quad(c[(1, 0, -1)], c[(-1, 0, -1)], c[(-1, 1, -1)], c[(1, 1, -1)])    # -z
    tris += _quad(c[(1, 0, 1)], c[(1, 0, -1)], c[(1, 1, -1)], c[(1, 1, 1)])        # +x
    tris += _quad(c[(-1, 0, -1)], c[(-1, 0, 1)], c[(-1, 1, 1)], c[(-1, 1, -1)])    # -x
    return tris


def cornell_box(width=256, height=256, light_size=0.5, light_emission=15.0, occluder=False, packer=None):
    """The procedural Cornell box (36 triangles; 48 with the occluder variant)."""
    s = Scene()
    s.name = "cornell_box"
    s.width, s.height = width, height
    tris, mats = [], []
    # walls: floor, ceiling, back (white = material 0), left (red = 1), right (green = 2); inward facing
    walls = [
        (_quad((-1, 0, -1), (-1, 0, 1), (1, 0, 1), (1, 0, -1)), 0),
        (_quad((-1, 2, -1), (1, 2, -1), (1, 2, 1), (-1, 2, 1)), 0),
        (_quad((-1, 0, -1), (1, 0, -1), (1, 2, -1), (-1, 2, -1)), 0),
        (_quad((-1, 0, -1), (-1, 2, -1), (-1, 2, 1), (-1, 0, 1)), 1),
        (_quad((1, 0, -1), (1, 0, 1), (1, 2, 1), (1, 2, -1)), 2),
    ]
    for q, m in walls:
        tris += q
        mats += [m, m]
    h = light_size / 2.0
    ly = 1.999
    if occluder:
        # emitter pushed into a recess above an occluding plate, so light reaches the room indirectly
        tris += _quad((-0.1, ly, -0.1), (0.1, ly, -0.1), (0.1, ly, 0.1), (-0.1, ly, 0.1))
        mats += [3, 3]
        tris += _quad((-0.35, 1.85, -0.35), (-0.35, 1.85, 0.35), (0.35, 1.85, 0.35), (0.35, 1.85, -0.35))
        mats += [0, 0]
        tris += _quad((-0.35, 1.80, -0.35), (0.35, 1.80, -0.35), (0.35, 1.80, 0.35), (-0.35, 1.80, 0.35))
        mats += [0, 0]
    else:
        tris += _quad((-h, ly, -h), (h, ly, -h), (h, ly, h), (-h, ly, h))
        mats += [3, 3]
    tb = _box((-0.35, 0.0, -0.3), (0.6, 1.2, 0.6), 17.0)
    tris += tb
    mats += [4] * 12
    sb = _box((0.4, 0.0, 0.35), (0.6, 0.6, 0.6), -17.0)
    tris += sb
    mats += [5] * 12
    v = np.asarray(tris, dtype=np.float32).reshape(-1, 3)
    s.blas.append({"vertices": v, "indices": None, "flags": 1})
    s.instances.append({"transform": IDENTITY.copy(), "blas": 0, "material_indices": np.asarray(mats, np.uint32)})
    s.diffuse = [solid((186, 186, 186, 255)), solid((165, 20, 20, 255)), solid((30, 140, 38, 255)),
                 solid((255, 255, 255, 255))]
    s.emission = [solid((255, 255, 255, 255))]
    s.attributes = [solid((77, 77, 0, 0))]  # roughness 0.3 in x/y
    s.materials = [
        _mat(0, packer=packer), _mat(1, packer=packer), _mat(2, packer=packer),
        _mat(3, emission=0, scale=light_emission if not occluder else light_emission * 6.25, packer=packer),
        _mat(0, attributes=0, ty=MaterialType.Metallic, packer=packer),
        _mat(3, ior=(1.5, 1.5), ty=MaterialType.Transparent, packer=packer),
    ]
    s.camera = make_camera((0.0, 1.0, 3.4), (0.0, 1.0, 0.0), 40.0, width / height, packer=packer)
    return s


def occluded_cornell(width=256, height=256, packer=None):
    return cornell_box(width, height, light_size=0.2, occluder=True, packer=packer)


def textured_cornell(width=128, height=128, glass_ior=(1.40, 1.75), seed=7, packer=None):
    """The Cornell geometry with every shading input non-uniform, so that the material decode of
    ray_hit (general.wesl:1086-1134) and the IOR pick of the quality hooks are exercised:

      * value-noise diffuse layers of different, non-square sizes; UVs per material that reach past
        [0, 1] (clamp-to-edge addressing); a recolour texture of random texels;
      * a noise emission texture on the ceiling light (emissive scale 15) and a wall that emits its
        own diffuse colour (diffuse scale 0.4);
      * noise attribute textures: the metal box's roughness and coat roughness vary over its faces,
        and the glass box is rough;
      * glass with a wide IOR range (per-path pick in Medium, dispersion in High) and a back wall
        that is diffuse with an IOR range (the Fresnel choice of general.wesl:735-751 at a diffuse
        vertex);
      * a noise cube-map sky behind the open front of the box.
    """
    rng = np.random.default_rng(seed)
    s = cornell_box(width, height, packer=packer)
    s.name = "textured_cornell"
    back = s.instances[0]["material_indices"].copy()
    back[4:6] = 6  # the back wall's two triangles (floor, ceiling, back, left, right: two each)
    s.instances[0]["material_indices"] = back

    def noise(h, w, lo=0.0, hi=1.0, alpha=None):
        n = value_noise(rng, max(h, w), octaves=3, base=4)[:h, :w]
        img = (np.clip(lo + (hi - lo) * n, 0.0, 1.0) * 255).astype(np.uint8)
        if alpha is not None:
            img[..., 3] = alpha
        return img

    s.diffuse = [noise(64, 64, 0.3, 0.9, 255), noise(48, 80, 0.1, 0.8, 255), noise(96, 32, 0.1, 0.8, 255),
                 noise(16, 16, 0.8, 1.0, 255)]
    s.emission = [noise(32, 32, 0.4, 1.0, 255)]
    att_metal = noise(64, 64)
    att_metal[..., 0:2] = (np.clip(0.05 + 0.55 * att_metal[..., 0:2] / 255.0, 0, 1) * 255).astype(np.uint8)
    att_metal[..., 2:4] = (0.3 * att_metal[..., 2:4]).astype(np.uint8)
    att_glass = noise(32, 48)
    att_glass[..., 0:2] = (np.clip(0.02 + 0.25 * att_glass[..., 0:2] / 255.0, 0, 1) * 255).astype(np.uint8)
    att_glass[..., 2:4] = 0
    s.attributes = [att_metal, att_glass]
    s.recolour = (rng.uniform(0.5, 1.0, (8, 8, 4)) * 255).astype(np.uint8)
    s.recolour[..., 3] = 255

    def uv3():
        return tuple(tuple(float(x) for x in rng.uniform(-0.2, 1.2, 2)) for _ in range(3))

    pk = _packer(packer)
    M = lambda d, e, a, es, ior, ty, rec=(0, 0): pk.material(*uv3(), rec, d, e, a, es, ior, ty)
    s.materials = [
        M(0, None, None, EmissionScale(0.0, 0.0), None, MaterialType.Diffuse, (1, 2)),
        M(1, None, None, EmissionScale(0.0, 0.0), None, MaterialType.Diffuse, (5, 3)),
        M(2, None, None, EmissionScale(0.0, 0.4), None, MaterialType.Diffuse, (7, 7)),
        M(3, 0, None, EmissionScale(15.0, 0.0), None, MaterialType.Diffuse),
        M(0, None, 0, EmissionScale(0.0, 0.0), (1.3, 1.6), MaterialType.Metallic, (2, 6)),
        M(3, None, 1, EmissionScale(0.0, 0.0), glass_ior, MaterialType.Transparent),
        M(0, None, None, EmissionScale(0.0, 0.0), (1.3, 1.5), MaterialType.Diffuse, (4, 1)),
    ]
    S = 32
    sky = np.zeros((6, S, S, 4), np.uint8)
    for f in range(6):
        sky[f] = noise(S, S, 0.05, 0.6 if f != 2 else 1.0, 255)
    s.sky = sky
    return s


# ---------------------------------------------------------------- icospheres
def icosphere(subdiv):
    t = (1.0 + 5 ** 0.5) / 2.0
    v = np.array([(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
                  (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)], dtype=np.float64)
    f = np.array([(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
                  (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5),
                  (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)], dtype=np.int64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    for _ in range(subdiv):
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        e.sort(axis=1)
        ue, inv = np.unique(e, axis=0, return_inverse=True)
        inv = inv.reshape(-1)
        mid = v[ue[:, 0]] + v[ue[:, 1]]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        base = v.shape[0]
        v = np.concatenate([v, mid])
        nf = f.shape[0]
        a, b, c = f[:, 0], f[:, 1], f[:, 2]
        ab, bc, ca = inv[:nf] + base, inv[nf:2 * nf] + base, inv[2 * nf:] + base
        f = np.concatenate([np.stack([a, ab, ca], 1), np.stack([b, bc, ab], 1), np.stack([c, ca, bc], 1),
                            np.stack([ab, bc, ca], 1)])
    return v, f


def random_rotation(rng):
    u1, u2, u3 = rng.random(3)
    q = np.array([math.sqrt(1 - u1) * math.sin(2 * math.pi * u2), math.sqrt(1 - u1) * math.cos(2 * math.pi * u2),
                  math.sqrt(u1) * math.sin(2 * math.pi * u3), math.sqrt(u1) * math.cos(2 * math.pi * u3)])
    x, y, z, w = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def _interp_matrix(size, g):
    """(size, g + 1) smoothstep-bilinear weights of lattice points for each pixel row."""
    coords = np.arange(size, dtype=np.float64) * (g / size)
    i0 = np.floor(coords).astype(np.int64)
    fr = coords - i0
    fr = fr * fr * (3 - 2 * fr)
    m = np.zeros((size, g + 1), np.float32)
    m[np.arange(size), i0] = 1 - fr
    m[np.arange(size), i0 + 1] += fr
    return m


def value_noise(rng, size, octaves=4, base=8, channels=4):
    """Fractal value noise in [0, 1): per octave, a random lattice interpolated as Wy @ L @ Wx^T."""
    out = np.zeros((channels, size, size), np.float32)
    amp, total = 1.0, 0.0
    for o in range(octaves):
        g = base << o
        lat = rng.random((channels, g + 1, g + 1)).astype(np.float32)
        w = _interp_matrix(size, g)
        out += amp * np.matmul(np.matmul(w, lat), w.T)
        total += amp
        amp *= 0.5
    return np.ascontiguousarray((out / total).transpose(1, 2, 0))


def icosphere_field(width=1920, height=1080, instances=64, subdiv=5, tex_size=1024, tex_layers=16, seed=2024,
                    packer=None):
    rng = np.random.default_rng(seed)
    s = Scene()
    s.name = f"icosphere_field_{instances}x{20 * 4 ** subdiv}"
    s.width, s.height = width, height
    base_v, faces = icosphere(subdiv)
    idx = faces.astype(np.uint32).reshape(-1)
    ntri = faces.shape[0]
    # textures: value noise; attribute x/y roughness in [0.05, 1], z/w coat roughness in [0, 0.3]
    for _ in range(tex_layers):
        s.diffuse.append((np.clip(0.15 + 0.8 * value_noise(rng, tex_size), 0, 1) * 255).astype(np.uint8))
        s.diffuse[-1][..., 3] = 255
        s.emission.append((np.clip(0.5 + 0.5 * value_noise(rng, tex_size), 0, 1) * 255).astype(np.uint8))
        r0 = rng.uniform(0.05, 1.0)
        n = value_noise(rng, tex_size)
        att = np.empty_like(n)
        att[..., 0:2] = np.clip(r0 + 0.1 * (n[..., 0:2] - 0.5), 0.05, 1.0)
        att[..., 2:4] = 0.3 * n[..., 2:4]
        s.attributes.append((att * 255).astype(np.uint8))
    kinds = rng.random(instances)
    n_variants = 8
    emissive_seen = False
    for i in range(instances):
        r = rng.uniform(1.2, 2.2)
        waves = [(rng.normal(size=3) * rng.uniform(1.0, 4.0), rng.uniform(0, 2 * math.pi), rng.uniform(0.02, 0.08))
                 for _ in range(6)]
        disp = np.ones(base_v.shape[0])
        for k, ph, amp in waves:
            disp += amp * np.sin(base_v @ k + ph)
        v = (base_v * (r * disp)[:, None]).astype(np.float32)
        s.blas.append({"vertices": v, "indices": idx, "flags": 1})
        R = random_rotation(rng)
        t = rng.uniform(-10.0, 10.0, 3)
        xf = np.concatenate([R, t[:, None]], axis=1).reshape(-1).astype(np.float32)
        kind = kinds[i]
        if kind < 0.02 or (i == instances - 1 and not emissive_seen):
            ty, ior, emis, scale = MaterialType.Diffuse, None, int(rng.integers(tex_layers)), float(np.exp(rng.normal(1, 1)))
            emissive_seen = True
        elif kind < 0.12:
            n0 = rng.uniform(1.3, 1.7)
            ty, ior, emis, scale = MaterialType.Transparent, (n0, n0 + 0.02), None, 1.0
        elif kind < 0.45:
            ty, ior, emis, scale = MaterialType.Metallic, None, None, 1.0
        else:
            ty, ior, emis, scale = MaterialType.Diffuse, None, None, 1.0
        first = len(s.materials)
        d_layer = int(rng.integers(tex_layers))
        a_layer = int(rng.integers(tex_layers))
        for _ in range(n_variants):
            uv = tuple(tuple(float(x) for x in rng.random(2)) for _ in range(3))
            s.materials.append(_mat(d_layer, emission=emis, attributes=a_layer, scale=scale, ior=ior, ty=ty, uv=uv,
                                    packer=packer))
        h = (np.arange(ntri, dtype=np.uint64) * np.uint64(2654435761) + np.uint64(i)) % np.uint64(n_variants)
        s.instances.append({"transform": xf, "blas": i, "material_indices": (first + h).astype(np.uint32)})
    # sky: vertical gradient on all six faces (bright above, dark below)
    S = 64
    ys = np.linspace(0, 1, S, dtype=np.float32)
    faces_img = np.zeros((6, S, S, 4), np.uint8)
    for fidx in range(6):
        if fidx == 2:
            col = np.array([0.85, 0.9, 1.0])
            img = np.tile(col, (S, S, 1))
        elif fidx == 3:
            img = np.tile(np.array([0.05, 0.05, 0.06]), (S, S, 1))
        else:
            tt = ys[:, None, None]  # t = 0 at the top (tc = -y)
            img = np.tile((1 - tt) * np.array([0.8, 0.85, 1.0]) + tt * np.array([0.08, 0.08, 0.1]), (1, S, 1))
        faces_img[fidx, ..., :3] = (np.clip(img, 0, 1) * 255).astype(np.uint8)
        faces_img[fidx, ..., 3] = 255
    s.sky = faces_img
    s.camera = make_camera((0.0, 2.0, 16.0), (0.0, 0.0, 0.0), 55.0, width / height, packer=packer)
    return s


def box_field(n_tris, width=512, height=512, seed=0, packer=None):
    """Cornell box plus subdivided boxes filling it up to about n_tris triangles (batched requests)."""
    rng = np.random.default_rng(seed)
    s = cornell_box(width, height, packer=packer)
    s.name = f"box_field_{n_tris}"
    v = [s.blas[0]["vertices"]]
    mats = [s.instances[0]["material_indices"]]
    have = 36
    while have < n_tris:
        k = int(min(64, max(1, math.sqrt((n_tris - have) / 12))))
        c = rng.uniform(-0.8, 0.8, 3)
        c[1] = rng.uniform(0.05, 1.2)
        sz = rng.uniform(0.05, 0.3, 3)
        ang = rng.uniform(-45, 45)
        tris = []
        for a in range(k):
            for b in range(k):
                off = np.array([(a / k - 0.5) * sz[0], 0.0, (b / k - 0.5) * sz[2]])
                tris += _box(tuple(c + off), tuple(sz / k), ang)
        tv = np.asarray(tris, np.float32).reshape(-1, 3)
        v.append(tv)
        mats.append(np.full(tv.shape[0] // 3, rng.integers(0, 3), np.uint32))
        have += tv.shape[0] // 3
    s.blas[0]["vertices"] = np.concatenate(v)
    s.instances[0]["material_indices"] = np.concatenate(mats)
    return s


def unit_cube_scene(width=128, height=128, packer=None):
    """The reference test's unit-cube geometry (src/tests/mod.rs:52-167): 8 vertices, 8 triangles."""
    s = Scene()
    s.name = "unit_cube"
    s.width, s.height = width, height
    verts = np.array([[0, 0, 0, 0], [0, 0, 1, 0], [0, 1, 0, 0], [0, 1, 1, 0], [1, 0, 0, 0], [1, 0, 1, 0],
                      [1, 1, 0, 0], [1, 1, 1, 0]], np.float32)
    idx = np.array([0, 1, 2, 3, 2, 1, 0, 4, 1, 1, 5, 4, 0, 2, 4, 6, 4, 2, 2, 3, 6, 7, 6, 3], np.uint32)
    s.blas.append({"vertices": verts, "indices": idx, "flags": 1})
    s.instances.append({"transform": IDENTITY.copy(), "blas": 0, "material_indices": np.arange(8, dtype=np.uint32)})
    P = ((1.0, 1.0), (0.0, 1.0), (1.0, 0.0), (0.0, 0.0))
    D = (2.4063, 2.4922)
    W = (1.33, 1.3442)
    spec = [(P[0], P[1], P[2], 0, 0, 0, D, 0), (P[3], P[2], P[1], 0, 0, 0, D, 0), (P[0], P[2], P[1], 1, 1, None, None, 0),
            (P[1], P[3], P[2], 1, 1, None, None, 0), (P[2], P[3], P[0], 0, 0, 0, None, 1),
            (P[1], P[0], P[3], 0, 0, 0, None, 1), (P[0], P[1], P[2], 1, None, None, W, 2),
            (P[1], P[3], P[2], 1, None, None, W, 2)]
    for a, b, c, d, e, att, ior, ty in spec:
        s.materials.append(_packer(packer).material(a, b, c, (0, 0), d, e, att, EmissionScale.from_emission_scale(1.0),
                                                    ior, ty))
    s.diffuse = [solid((34, 177, 76, 255)), solid((250, 250, 250, 255))]
    s.emission = [solid((255, 0, 0, 255)), solid((0, 0, 0, 255))]
    s.attributes = [solid((20, 20, 0, 255))]
    s.camera = make_camera((2.5, 2.0, 2.5), (0.5, 0.5, 0.5), 45.0, width / height, packer=packer)
    return s


def with_spheres(s, n=48, seed=0, scale=0.9, angle_deg=30.0, offset=(0.1, 0.7, 0.0), material=0):
    """Adds an instance of procedural geometry: n axis-aligned cubes, each holding the sphere inscribed
    in it (radius = half the x extent), for an intersection handler such as tests/data/sphere_handler.cu.
    The instance is rotated about y, scaled uniformly and moved by `offset`."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(-0.6, 0.6, (n, 3))
    r = rng.uniform(0.04, 0.12, n)
    aabbs = np.concatenate([c - r[:, None], c + r[:, None]], axis=1).astype(np.float32)
    a = math.radians(angle_deg)
    ca, sa = math.cos(a) * scale, math.sin(a) * scale
    xf = np.array([ca, 0.0, sa, offset[0], 0.0, scale, 0.0, offset[1], -sa, 0.0, ca, offset[2]], np.float32)
    s.blas.append({"aabbs": aabbs, "flags": 1})
    s.instances.append({"transform": xf, "blas": len(s.blas) - 1,
                        "material_indices": np.full(n, material, np.uint32)})
    return s
