"""State of the compression density regularisation
(``tensorsph.compression_regularization``): the rule, the normalisation and
the global inverse reference compression that one ``rhs`` call uses and the
next one receives (compression_regularization.py:192-240).  The arithmetic
runs inside the 2-D ``rhs`` on the device (``csrc/wcsph.cu``)."""
from __future__ import annotations

RULES = ("internal", "free_surface", "free_stream")
NORMALIZATIONS = ("reference_mean", "none")

__all__ = ["RULES", "NORMALIZATIONS", "CompressionRegularization"]


class CompressionRegularization:
    """The scalar state carried between steps in ``rhs(..., state=...)``
    under ``state["compression"]``; ``inverse_reference_compression`` starts
    at 1 and holds 1 / mean{S_i : S_i > 1} of the last call."""

    def __init__(self, rule: str = "free_surface", normalization: str = "reference_mean") -> None:
        if rule not in RULES:
            raise ValueError(f"unknown rule {rule!r}; expected one of {RULES}")
        if normalization not in NORMALIZATIONS:
            raise ValueError(f"unknown normalization {normalization!r}; expected one of {NORMALIZATIONS}")
        self.rule = rule
        self.normalization = normalization
        self.inverse_reference_compression = 1.0
