"""gs.textures (options/textures.py): the texture options a surface can carry.  There is no
renderer in this build, so they are kept as plain option records for scripts that pass them
to gs.surfaces; nothing reads images."""

from __future__ import annotations

from .exceptions import GenesisException


class Texture:
    def __init__(self, **kw):
        for k, v in kw.items():
            setattr(self, k, v)


class ColorTexture(Texture):
    """A single color (options/textures.py:40-76)."""

    def __init__(self, color=(1.0, 1.0, 1.0), **kw):
        super().__init__(**kw)
        self.color = (float(color),) if isinstance(color, (int, float)) else tuple(float(c) for c in color)
        if any(not 0.0 <= c <= 1.0 for c in self.color):
            raise GenesisException("Color values must be within [0, 1].")


class ImageTexture(Texture):
    """An image file (options/textures.py:78-): the path and options are recorded, the image is
    not loaded."""

    def __init__(self, image_path=None, image_array=None, image_color=None, encoding="srgb", **kw):
        super().__init__(**kw)
        if image_path is None and image_array is None:
            raise GenesisException("Either `image_path` or `image_array` must be provided.")
        self.image_path, self.image_array, self.image_color, self.encoding = image_path, image_array, image_color, encoding


__all__ = ["Texture", "ColorTexture", "ImageTexture"]
