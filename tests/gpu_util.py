"""Small helpers for the GPU parity tests (numpy <-> CUDA tensors with the library's layouts)."""
import numpy as np
import torch


def dev(a):
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint32:
        a = a.view(np.int32)
    elif a.dtype == np.uint64:
        a = a.view(np.int64)
    return torch.from_numpy(a).cuda()


def host(t, dtype=None):
    a = t.detach().cpu().numpy()
    if dtype is not None:
        a = a.view(dtype)
    return a


def counts(t):
    torch.cuda.synchronize()
    return host(t, np.uint32)


class SceneOnDevice:
    def __init__(self, sc):
        self.sc = sc
        self.faces = dev(sc.faces)
        self.edges = dev(sc.edges)
        self.body = dev(sc.body)
        self.d_hat = dev(sc.d_hat)
        self.offset = dev(sc.offset)
        self.vert_area = dev(sc.vert_area)
        self.face_area = dev(sc.face_area)
        self.edge_area = dev(sc.edge_area)
