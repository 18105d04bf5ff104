"""tc_b200 -- B200-native operator application (HF exchange and the
transcorrelated two- and three-body terms) behind TC++'s calc_hamiltonian
interface.  See include/tcg.h for the C-ABI."""
from . import abi  # noqa: F401
from . import synth  # noqa: F401
from ._lib import TCError  # noqa: F401
from .context import Context, sum_of_vaux  # noqa: F401
from .system import TCSystem  # noqa: F401

__all__ = ["abi", "synth", "TCError", "Context", "sum_of_vaux", "TCSystem"]
