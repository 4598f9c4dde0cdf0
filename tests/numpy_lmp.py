"""lmp-like vectors and CSR matrices on host memory over the CPU oracle --
TEST INFRASTRUCTURE ONLY: lets the multi-rank host logic of ba_b200.coupled
run in gloo / thread ranks on CPU without a GPU."""
import numpy as np

import oracle


class NumpyVector:
    def __init__(self, n):
        self.a = np.zeros(n)

    def GetValues(self, idx):
        return self.a[np.asarray(idx)].copy()

    def SetValues(self, idx, values):
        self.a[np.asarray(idx)] = values

    def Dot(self, other):
        return oracle.dot(self.a, other.a) if self.a.size else 0.0

    def Axpy(self, other, s):
        self.a += s * other.a

    def ScaleAdd(self, s, other):
        self.a = s * self.a + other.a

    def CopyFrom(self, other):
        self.a[:] = other.a

    def Zeros(self):
        self.a[:] = 0.0

    def ElementWiseMult(self, other):
        self.a *= other.a


class NumpyCSR:
    def __init__(self, rp, c, v, ncol):
        self.rp, self.c, self.v, self.ncol = (np.asarray(rp, np.int32), np.asarray(c, np.int32),
                                              np.asarray(v, np.float64), ncol)

    def VectorMult(self, x, y):
        y.a[:] = oracle.spmv(self.rp, self.c, self.v, x.a)

    def VectorMultAdd(self, x, y):
        y.a += oracle.spmv(self.rp, self.c, self.v, x.a)

    def extract_invdiagelements(self, vec):
        vec.a[:] = oracle.invdiag(self.rp, self.c, self.v)


def numpy_backend():
    return (lambda rp, c, v, ncol: NumpyCSR(rp, c, v, ncol)), (lambda n: NumpyVector(n))
