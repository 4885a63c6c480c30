"""Single-rank stand-in for mpi4py, used only to import the reference
qttools package in the container that generates the golden fixtures
(mpi4py is not installed there). Every collective is the identity on one
rank."""
