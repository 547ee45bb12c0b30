"""tigerci_b200 - B200-native sigma-vector build (sigma = H c) for TigerCI's
multireference singles-and-doubles CI, behind a C ABI (include/tigerci_sigma.h)."""
from .api import KILL_NUMBER, CsfSpace, Deck, Operator, Plan, SigmaBuilder, aposteriori  # noqa: F401

__all__ = ["Deck", "CsfSpace", "Operator", "Plan", "SigmaBuilder", "KILL_NUMBER"]
