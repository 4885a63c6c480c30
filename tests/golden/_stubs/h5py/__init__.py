"""Empty stand-in: the reference imports h5py at module level for HDF5
input loading, which the GF-solver path never calls."""


class File:  # pragma: no cover - never used on the solver path
    def __init__(self, *args, **kwargs):
        raise RuntimeError("h5py stand-in: HDF5 I/O is unavailable")
