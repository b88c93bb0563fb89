"""``pyfourier_b200.pipemenon.pipe_menon_dcf``: the module path of the reference's
``pyfourier.pipemenon`` (src/pyfourier/__init__.py:15, :41)."""

from ._dcf import pipe_menon_dcf

__all__ = ["pipe_menon_dcf"]
