"""gs.surfaces: the visual description of an entity (genesis/options/surfaces.py).  There is
no renderer on this path, so a surface is only recorded on its entity (scripts written for
Genesis pass one to add_entity); its fields keep the reference's names and defaults."""

from __future__ import annotations

from .exceptions import GenesisException

_VIS_MODES = (None, "visual", "particle", "sdf", "collision", "recon")


class Surface:
    _defaults = dict(color=None, opacity=None, roughness=None, metallic=None, emissive=None, ior=None,
                     vis_mode=None, smooth=True, double_sided=None, cutoff=180.0, normal_diff_clamp=180.0,
                     recon_backend="splashsurf", generate_foam=False, foam_options=None, default_roughness=1.0)

    def __init__(self, **data):
        fields = {}
        for klass in reversed(type(self).__mro__):
            fields.update(getattr(klass, "_defaults", {}))
        for k, v in data.items():
            if k not in fields and not k.endswith("_texture"):
                raise GenesisException(f"Unrecognized attribute: {k} for {type(self).__name__}")
        for k, v in fields.items():
            setattr(self, k, data.get(k, v))
        for k, v in data.items():
            if k.endswith("_texture"):
                setattr(self, k, v)
        if self.vis_mode not in _VIS_MODES:
            raise GenesisException(f"Unsupported vis_mode: {self.vis_mode}")

    def __repr__(self):
        return f"<gs.surfaces.{type(self).__name__}(color={self.color}, vis_mode={self.vis_mode})>"


class Glass(Surface):
    _defaults = dict(roughness=0.0, ior=1.5, subsurface=False, thickness=None)


class Water(Glass):
    _defaults = dict(color=(0.61, 0.98, 0.93), roughness=0.2, ior=1.2)


class Metal(Surface):
    _defaults = dict(roughness=0.1, metal_type="iron")


class Iron(Metal):
    _defaults = dict(metal_type="iron")


class Aluminium(Metal):
    _defaults = dict(metal_type="aluminium")


class Copper(Metal):
    _defaults = dict(metal_type="copper")


class Gold(Metal):
    _defaults = dict(metal_type="gold")


class Plastic(Surface):
    _defaults = dict(ior=1.0)


class Rough(Plastic):
    _defaults = dict(roughness=1.0, ior=1.5)


class Smooth(Plastic):
    _defaults = dict(roughness=0.1, ior=1.5)


class Reflective(Plastic):
    _defaults = dict(roughness=0.01, ior=2.0)


class Collision(Plastic):
    _defaults = dict(color=(0.5, 0.5, 0.5))


class BSDF(Surface):
    _defaults = dict(specular_trans=0.0, diffuse_trans=0.0)


class Default(BSDF):
    pass


class Emission(Surface):
    pass


__all__ = ["Surface", "Default", "Glass", "Water", "Metal", "Iron", "Aluminium", "Copper", "Gold", "Plastic",
           "Rough", "Smooth", "Reflective", "Collision", "BSDF", "Emission"]
