"""Error type raised by the public API (genesis/__init__.py: gs.GenesisException)."""


class GenesisException(Exception):
    pass
