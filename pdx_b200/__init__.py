"""B200-native search engine for the PDX vector layout (cwida/PDX search path)."""
from .index_factory import (IndexPDXIVF, IndexPDXIVFSQ8, IndexPDXIVFTree, IndexPDXIVFTreeSQ8,
                            load_index)

__all__ = ["IndexPDXIVF", "IndexPDXIVFSQ8", "IndexPDXIVFTree", "IndexPDXIVFTreeSQ8", "load_index"]
