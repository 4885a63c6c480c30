"""Single-rank MPI stand-in (see package docstring)."""
import numpy as _np

SUM = "sum"
PROD = "prod"
MAX = "max"
MIN = "min"
LAND = "land"
LOR = "lor"
IN_PLACE = object()


def Get_library_version():
    return "single-rank stub"


class Request:
    @staticmethod
    def Waitall(requests):
        return None

    def Wait(self):
        return None


class Comm:
    rank = 0
    size = 1

    def Get_rank(self):
        return 0

    def Get_size(self):
        return 1

    def Get_info(self):
        return {}

    def Split(self, color=0, key=0):
        return Comm()

    def Barrier(self):
        return None

    barrier = Barrier

    def bcast(self, obj, root=0):
        return obj

    def allgather(self, obj):
        return [obj]

    def gather(self, obj, root=0):
        return [obj]

    def allreduce(self, obj, op=SUM):
        return obj

    def _copy(self, sendbuf, recvbuf):
        if sendbuf is IN_PLACE or recvbuf is None:
            return
        src = sendbuf[0] if isinstance(sendbuf, (list, tuple)) else sendbuf
        dst = recvbuf[0] if isinstance(recvbuf, (list, tuple)) else recvbuf
        _np.copyto(_np.asarray(dst).reshape(-1), _np.asarray(src).reshape(-1))

    def Allreduce(self, sendbuf, recvbuf, op=SUM):
        self._copy(sendbuf, recvbuf)

    def Allgather(self, sendbuf, recvbuf):
        self._copy(sendbuf, recvbuf)

    def Alltoall(self, sendbuf, recvbuf):
        self._copy(sendbuf, recvbuf)

    def Bcast(self, buf, root=0):
        return None

    def Free(self):
        return None


Intracomm = Comm
COMM_WORLD = Comm()
