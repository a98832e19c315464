"""multem_b200 — B200-native multislice engine with MULTEM's input/output conventions."""
from .input import Parameters, SystemConf  # noqa: F401
