"""Textures of the scene API (``liar.textures``, src/liar/textures/).

On the GPU path: Constant (textures/constant.cpp), a spectrum or a number; and the uv textures
CheckerBoard (checker_board.cpp), GridBoard (grid_board.cpp), TransformationUv
(transformation_uv.cpp) and Image (image.cpp), which pick, move between or look up colours by
the hit's (u, v) coordinates. A material parameter that is a uv texture becomes a tree of liar_texture nodes
(include/liar_gpu.h) that the kernels walk at every hit; emission and roughness slots take
constant textures only."""
from __future__ import annotations

import warnings

import math

import numpy as np

from .spectra import Spectrum


class Texture:
    pass


class Constant(Texture):
    def __init__(self, value=1.0):
        self.value = value if isinstance(value, Spectrum) else Spectrum(float(value))

    @property
    def spectrum(self) -> Spectrum:
        return self.value


def _texture(x) -> Texture:
    """A texture slot's value as a texture: textures as they are, spectra and numbers as Constant."""
    if isinstance(x, Texture):
        return x
    if isinstance(x, (Spectrum, int, float)):
        return Constant(x)
    raise TypeError(f"expected a texture, a spectrum or a number, got {type(x).__name__}")


class BinaryOperator(Texture):
    """Base of the textures that mix two inputs (binary_operator.cpp): textureA, textureB."""

    def __init__(self, a, b):
        self.textureA = _texture(a)
        self.textureB = _texture(b)


class UnaryOperator(Texture):
    """Base of the textures with one input (unary_operator.cpp): texture."""

    def __init__(self, texture):
        self.texture = _texture(texture)


class CheckerBoard(BinaryOperator):
    """CheckerBoard(a, b): a where the fractional u and v lie on the same side of ``split``
    (default (0.5, 0.5)), else b (checker_board.cpp:113-207).

    antiAliasing "none" is the reference's point lookup. "bilinear" (the reference's default)
    blends a and b by a's share of the pixel footprint that the camera's ray differentials give
    (CheckerBoard::integrate); hits without differentials (past the camera vertex) look up the
    point."""

    AA_NONE = "none"
    AA_BILINEAR = "bilinear"
    _default_aa = "bilinear"

    def __init__(self, a, b):
        super().__init__(a, b)
        self.split = (0.5, 0.5)
        self.antiAliasing = CheckerBoard._default_aa

    @property
    def split(self):
        return self._split

    @split.setter
    def split(self, value):
        u, v = value
        self._split = (float(u), float(v))

    @property
    def antiAliasing(self) -> str:
        return self._aa

    @antiAliasing.setter
    def antiAliasing(self, mode: str):
        mode = str(mode).lower()
        if mode not in (self.AA_NONE, self.AA_BILINEAR):
            raise KeyError(f"antiAliasing must be 'none' or 'bilinear', not {mode!r}")
        self._aa = mode

    @staticmethod
    def setDefaultAntiAliasing(mode: str):
        mode = str(mode).lower()
        if mode not in (CheckerBoard.AA_NONE, CheckerBoard.AA_BILINEAR):
            raise KeyError(f"antiAliasing must be 'none' or 'bilinear', not {mode!r}")
        CheckerBoard._default_aa = mode


class GridBoard(BinaryOperator):
    """GridBoard(a, b): a on grid lines of ``thickness`` (default (0.1, 0.1)) around the integer u
    and v, else b. As in grid_board.cpp:80-87, the first thickness bounds u at both sides and v
    from below, the second v from above."""

    def __init__(self, a, b):
        super().__init__(a, b)
        self.thickness = (0.1, 0.1)

    @property
    def thickness(self):
        return self._thickness

    @thickness.setter
    def thickness(self, value):
        u, v = value
        self._thickness = (float(u), float(v))


def as_matrix2d(m) -> np.ndarray:
    """A 3 x 3 float64 matrix of a 2D affine transformation: 3 x 3 or 2 x 3 (row-major, the last
    column the translation), 9 or 6 numbers, or an object with a `matrix` attribute."""
    if hasattr(m, "matrix"):
        m = m.matrix
    a = np.asarray(m, dtype=np.float64)
    if a.size == 9:
        a = a.reshape(3, 3)
    elif a.size == 6:
        a = np.vstack([a.reshape(2, 3), [0.0, 0.0, 1.0]])
    else:
        raise ValueError("a 2D transformation is a 3 x 3 or 2 x 3 matrix")
    if not np.allclose(a[2], [0.0, 0.0, 1.0]):
        raise NotImplementedError("projective uv transformations are not on the GPU path")
    return a


class TransformationUv(UnaryOperator):
    """TransformationUv(texture, transformation): texture looked up at the transformed (u, v)
    (transformation_uv.cpp:67-70)."""

    def __init__(self, texture, transformation):
        super().__init__(texture)
        self.transformation = transformation

    @property
    def transformation(self) -> np.ndarray:
        return self._matrix

    @transformation.setter
    def transformation(self, value):
        self._matrix = as_matrix2d(value)


def _mip_compress(level: np.ndarray, axis: int, new_size: int) -> np.ndarray:
    """Image::makeMipMap (image.cpp:428-560): one level halved along axis (1 = x, 0 = y) of an
    (h, w, 4) float32 level. An even size averages pairs; an odd size 2 n + 1 weighs three
    neighbours (n - k, n, k + 1) / (2 n + 1). Along x the weights are those of the reference's
    vectorised build (the default, LIAR_HAVE_AVX), which multiplies the middle pixel by itself
    instead of by its weight (image.cpp:528-531); along y it uses the weight. A zero size keeps
    the parent."""
    old = level.shape[axis]
    if new_size == 0 or level.shape[1 - axis] == 0:
        return level
    a = np.moveaxis(level, axis, 0)
    if 2 * new_size == old:
        out = (a[0::2] + a[1::2]) * np.float32(0.5)
    else:
        if 2 * new_size + 1 != old:
            raise ValueError("mip level sizes must halve")
        scale = np.float32(1.0) / np.float32(old)
        k = np.arange(new_size, dtype=np.float32)
        w0 = (scale * (np.float32(new_size) - k))[:, None, None]
        w1 = scale * np.float32(new_size)
        w2 = (scale * (k + np.float32(1)))[:, None, None]
        p0, p1, p2 = a[0:2 * new_size:2], a[1:2 * new_size:2], a[2:2 * new_size + 1:2]
        mid = p1 * p1 if axis == 1 else w1 * p1
        out = (w0 * p0 + mid) + w2 * p2
    return np.ascontiguousarray(np.moveaxis(out.astype(np.float32), 0, axis))


def mip_levels(pixels: np.ndarray, mode: str) -> tuple[int, int, list]:
    """Image::makeMipMaps (image.cpp:365-425): (levels along u, levels along v, [levels]) of an
    (h, w, 4) image, level (iu, iv) at index iv * levels_u + iu. "none": the image alone;
    "isotropic": floor(log2(max(w, h))) + 1 levels, each halving x then y; "anisotropic":
    (floor(log2 w) + 1) x (floor(log2 h) + 1) levels, row iv the image halved iv times along y and
    then iu times along x."""
    h, w = pixels.shape[:2]
    base = np.ascontiguousarray(pixels, dtype=np.float32)
    if mode == Image.MM_NONE:
        return 1, 1, [base]
    if mode == Image.MM_ISOTROPIC:
        n = int(math.floor(math.log2(max(w, h)))) + 1
        levels = [base]
        for i in range(1, n):
            tmp = _mip_compress(levels[-1], 1, w >> i)
            levels.append(_mip_compress(tmp, 0, h >> i))
        return n, 1, levels
    nu, nv = int(math.floor(math.log2(w))) + 1, int(math.floor(math.log2(h))) + 1
    levels = [base]
    for j in range(nv):
        if j > 0:
            levels.append(_mip_compress(levels[(j - 1) * nu], 0, h >> j))
        for i in range(1, nu):
            levels.append(_mip_compress(levels[-1], 1, w >> i))
    return nu, nv, levels


def image_pool_block(t) -> np.ndarray:
    """The texture_pixels block of an image texture (include/liar_gpu.h, LIAR_TEX_IMAGE): the mip
    table's header {levels u, levels v, mip mode, 0} and one entry {offset low 31 bits, offset
    high bits, width, height} per level, as int32 bits in float32, then every level's pixels."""
    px = np.zeros(t.xyz.shape[:2] + (4,), np.float32)
    px[..., :3] = t.xyz
    nu, nv, levels = mip_levels(px, t.mipMapping)
    head = np.zeros((1 + nu * nv, 4), np.int32)
    head[0] = (nu, nv, {Image.MM_NONE: 0, Image.MM_ISOTROPIC: 1, Image.MM_ANISOTROPIC: 2}[t.mipMapping], 0)
    off = 1 + nu * nv
    for k, lv in enumerate(levels):
        head[1 + k] = (off & 0x7FFFFFFF, off >> 31, lv.shape[1], lv.shape[0])
        off += lv.shape[0] * lv.shape[1]
    return np.concatenate([head.view(np.float32)] + [lv.reshape(-1, 4) for lv in levels])


class Image(Texture):
    """Image(path[, antiAliasing, mipMapping][, rgbSpace]) (textures/image.cpp): the picture read
    as XYZ (codecs.read) and looked up at (u, 1 - v) with wrap-around; its colour becomes a
    spectrum through the standard recovery (Spectral::fromXYZ).

    antiAliasing "none" takes the nearest pixel, "bilinear" blends the four around, "trilinear"
    (the reference's default) blends bilinear lookups of the two mip levels around the level that
    the camera's ray differentials' footprint picks (mipMapping "anisotropic", the default, per
    axis; "isotropic" by the larger; "none" always the image itself). Hits without differentials
    (past the camera vertex) look up level 0."""

    AA_NONE, AA_BILINEAR, AA_TRILINEAR = "none", "bilinear", "trilinear"
    MM_NONE, MM_ISOTROPIC, MM_ANISOTROPIC = "none", "isotropic", "anisotropic"
    _default_aa = "trilinear"
    _default_mm = "anisotropic"

    def __init__(self, path=None, *args):
        aa, mm, space = Image._default_aa, Image._default_mm, None
        if len(args) == 1:
            space = args[0]
        elif len(args) >= 2:
            aa, mm = args[0], args[1]
            space = args[2] if len(args) > 2 else None
        self.antiAliasing = aa
        self.mipMapping = mm
        self.filename = None
        self.rgbSpace = None
        self.xyz = None
        if path is not None:
            self.loadFile(path, space)

    def loadFile(self, path, rgbSpace=None):
        from . import codecs
        xyza, space = codecs.read(path, rgbSpace)
        if xyza.shape[0] == 0 or xyza.shape[1] == 0:
            raise ValueError("bad image resolution")
        self.filename, self.rgbSpace = str(path), space
        self.xyz = np.ascontiguousarray(xyza[..., :3], dtype=np.float32)

    @classmethod
    def from_xyz(cls, xyz, antiAliasing="bilinear", mipMapping="none"):
        """An image texture of XYZ pixels (H, W, 3), row 0 at the top."""
        t = cls(None, antiAliasing, mipMapping)
        t.xyz = np.ascontiguousarray(np.asarray(xyz, dtype=np.float32).reshape(*np.shape(xyz)[:2], 3))
        return t

    @property
    def resolution(self):
        return (self.xyz.shape[1], self.xyz.shape[0]) if self.xyz is not None else (0, 0)

    @property
    def antiAliasing(self) -> str:
        return self._aa

    @antiAliasing.setter
    def antiAliasing(self, mode):
        mode = str(mode).lower()
        if mode not in (self.AA_NONE, self.AA_BILINEAR, self.AA_TRILINEAR):
            raise KeyError(f"antiAliasing must be 'none', 'bilinear' or 'trilinear', not {mode!r}")
        self._aa = mode

    @property
    def mipMapping(self) -> str:
        return self._mm

    @mipMapping.setter
    def mipMapping(self, mode):
        mode = str(mode).lower()
        if mode not in (self.MM_NONE, self.MM_ISOTROPIC, self.MM_ANISOTROPIC):
            raise KeyError(f"mipMapping must be 'none', 'isotropic' or 'anisotropic', not {mode!r}")
        self._mm = mode

    @staticmethod
    def setDefaultAntiAliasing(mode):
        Image._default_aa = str(mode).lower()

    @staticmethod
    def setDefaultMipMapping(mode):
        Image._default_mm = str(mode).lower()


_U32, _U64 = 0xFFFFFFFF, 0xFFFFFFFFFFFFFFFF
# PCG constants (O'Neill 2014, pcg-random.org): the default 64-bit and 32-bit LCG multipliers and
# increments, and the 32-bit MCG multiplier of the RXS M XS output with its inverse mod 2^32
_PCG_MUL64, _PCG_INC64 = 6364136223846793005, 1442695040888963407
_PCG_MUL32, _PCG_INC32 = 747796405, 2891336453
_RXS_MUL32, _RXS_UNMUL32 = 277803737, 2897767785


def _xsh_rs_64_32(state: int) -> int:
    """PCG's XSH RS output, 64-bit state to 32 bits: xorshift by 22, then a shift of 22 to 29
    chosen by the top 3 bits."""
    rshift = state >> 61
    state ^= state >> 22
    return (state >> (22 + rshift)) & _U32


def _rxs_m_xs_32(state: int) -> int:
    """PCG's RXS M XS output on 32 bits (a bijection): random xorshift, multiply, xorshift by 22."""
    state ^= state >> (4 + (state >> 28))
    state = (state * _RXS_MUL32) & _U32
    return state ^ (state >> 22)


def _unxorshift32(y: int, shift: int) -> int:
    x = y
    for _ in range(32 // shift + 1):
        x = y ^ (x >> shift)
    return x & _U32


def _rxs_m_xs_32_inverse(value: int) -> int:
    x = _unxorshift32(value, 22)
    x = (x * _RXS_UNMUL32) & _U32
    return _unxorshift32(x, 4 + (x >> 28))


class Pcg32K2Fast:
    """pcg32_k2_fast of pcg-cpp (O'Neill, "PCG: A Family of Simple Fast Space-Efficient
    Statistically Good Algorithms for Random Number Generation", 2014): a 64-bit one-stream LCG
    with the XSH RS output, extended by a 2-entry table of 32-bit values XORed into every output
    (entry picked by the state's low bit; the table advances, as a 32-bit RXS M XS generator run
    inside out, whenever the state's low 32 bits are all zero). The reference seeds one with the
    Perlin seed (src/liar/textures/perlin.cpp:140)."""

    def __init__(self, seed: int):
        self.state = (((seed & _U64) + _PCG_INC64) * _PCG_MUL64 + _PCG_INC64) & _U64
        # the table starts from the base generator's outputs, offset by the difference of two
        a, b = self._base(), self._base()
        diff = (a - b) & _U32
        self.table = [self._base() ^ diff for _ in range(2)]

    def _base(self) -> int:
        old = self.state
        self.state = (old * _PCG_MUL64 + _PCG_INC64) & _U64
        return _xsh_rs_64_32(old)

    def _advance_table(self) -> None:
        carry = False
        for i in range(len(self.table)):
            if carry:
                carry = self._step_entry(i)
            carry = self._step_entry(i) or carry

    def _step_entry(self, i: int) -> bool:
        st = _rxs_m_xs_32_inverse(self.table[i])
        st = (st * _PCG_MUL32 + _PCG_INC32 + 2 * (i + 1)) & _U32
        self.table[i] = _rxs_m_xs_32(st)
        return self.table[i] == 0

    def __call__(self) -> int:
        if (self.state & _U32) == 0:
            self._advance_table()
        ext = self.table[self.state & 1]
        return self._base() ^ ext


def _uniform_below(g, n: int) -> int:
    """A uniform integer in [0, n) from a 32-bit generator, as libstdc++'s
    uniform_int_distribution draws it: Lemire's multiply-and-reject ("Fast Random Integer
    Generation in an Interval", 2019) on a 64-bit product."""
    product = g() * n
    low = product & _U32
    if low < n:
        threshold = ((1 << 32) - n) % n
        while low < threshold:
            product = g() * n
            low = product & _U32
    return product >> 32


def std_shuffle(values: list, g) -> None:
    """std::shuffle of libstdc++ (GCC 11 and later) with a 32-bit generator: Fisher-Yates from the
    front, one draw per element, except that while i * (i + 1) fits the generator's range two
    positions come from one draw of [0, (i + 1)(i + 2)) (its quotient and remainder by i + 2), after
    a first single swap when the length is even."""
    n = len(values)
    if n < 2:
        return
    if (1 << 32) - 1 < n * n:
        raise NotImplementedError("ranges beyond the paired draws are not needed here")
    i = 1
    if n % 2 == 0:
        j = _uniform_below(g, 2)
        values[1], values[j] = values[j], values[1]
        i = 2
    while i < n:
        r = i + 1
        x = _uniform_below(g, r * (r + 1))
        a, b = x // (r + 1), x % (r + 1)
        values[i], values[a] = values[a], values[i]
        values[i + 1], values[b] = values[b], values[i + 1]
        i += 2


def perlin_tables(seed: int) -> np.ndarray:
    """The reference's three lattice permutation tables of Perlin(seed) (perlin.cpp:137-152): one
    pcg32_k2_fast seeded with the seed shuffles 0..255 for x, then y, then z; a padding entry
    repeats each table's first value. (3, 257) uint8."""
    g = Pcg32K2Fast(int(seed) & _U32)
    out = np.zeros((3, 257), np.uint8)
    for k in range(3):
        t = list(range(256))
        std_shuffle(t, g)
        out[k, :256] = t
        out[k, 256] = t[0]
    return out


class Perlin(Texture):
    """Perlin([seed]) (textures/perlin.cpp): improved Perlin noise of the hit point, a flat
    spectrum. The lattice's three permutation tables are the reference's for the same seed
    (perlin_tables: pcg32_k2_fast through libstdc++'s std::shuffle, as a Linux build of the
    reference draws them)."""

    def __init__(self, seed: int = 0):
        self.seed = int(seed)

    @property
    def seed(self) -> int:
        return self._seed

    @seed.setter
    def seed(self, value: int):
        self._seed = int(value) & 0xFFFFFFFF
        self.tables = perlin_tables(self._seed)


class FBm(Perlin):
    """FBm(numOctaves[, falloff]) (textures/fbm.cpp): octaves of Perlin noise (seed 0) at doubling
    frequencies, weighed by falloff^k (default 0.5). The reference lowers the octave count where
    the ray differentials' footprint is wide; this path has no differentials, so every octave
    counts (the reference's zero-footprint case)."""

    def __init__(self, numOctaves: int, falloff: float = 0.5):
        super().__init__(0)
        if int(numOctaves) < 1 or int(numOctaves) > 64:
            raise ValueError("numOctaves must be in 1..64")
        self.numOctaves = int(numOctaves)
        self.falloff = float(falloff)


class Abs(UnaryOperator):
    """Abs(texture) (textures/abs.cpp): the absolute value of its input."""


class Product(Texture):
    """Product(factors) or Product(a, b) (textures/product.cpp). On the GPU path at most one factor
    may vary; the others must be flat constants (numbers or constant spectra of one value)."""

    def __init__(self, *args):
        factors = args[0] if len(args) == 1 and isinstance(args[0], (list, tuple)) else args
        self.factors = [_texture(f) for f in factors]


class Sum(Texture):
    """Sum(terms) or Sum(a, b) (textures/sum.cpp). On the GPU path at most one term may vary; the
    others must be flat constants."""

    def __init__(self, *args):
        terms = args[0] if len(args) == 1 and isinstance(args[0], (list, tuple)) else args
        self.terms = [_texture(t) for t in terms]


def flat_value(t) -> float | None:
    """The value of a flat constant texture (a number or a constant spectrum), else None."""
    if isinstance(t, Constant) and type(t.value) is Spectrum:
        return float(t.value.value)
    return None


def is_uv_texture(x) -> bool:
    return isinstance(x, (CheckerBoard, GridBoard, TransformationUv, Image, Perlin, Abs, Product, Sum))


def as_spectrum(x) -> Spectrum:
    """Spectrum of a constant texture, a spectrum or a number (the texture slots that take
    constants only)."""
    if isinstance(x, Constant):
        return x.value
    if isinstance(x, Spectrum):
        return x
    if isinstance(x, (int, float)):
        return Spectrum(float(x))
    raise TypeError(f"unsupported texture {type(x).__name__} in this slot: it takes constant textures only")


def as_scalar(x) -> float:
    """Scalar of a texture slot that the shaders read with scalarLookUp (roughness)."""
    s = as_spectrum(x)
    if type(s) is Spectrum:
        return s.value
    raise TypeError("roughness textures must be flat")
