"""Save/load narrow-phase cases (inputs + reference outputs) as .npz files."""
import numpy as np

from reactphysics3d_b200 import _abi as A

PAIR_FIELDS = ("shape1", "shape2", "pos1", "rot1", "pos2", "rot2")
OUT_FIELDS = ("is_colliding", "nb_contacts", "normal_depth", "local1", "local2")


def pack_case(d, prefix, algo, pairs, out, cache_out=None, clip=True):
    d[prefix + "algo"] = np.array(algo)
    d[prefix + "clip"] = np.array(int(clip))
    for f in PAIR_FIELDS:
        d[prefix + f] = getattr(pairs, f)
    if pairs.report is not None:
        d[prefix + "report"] = pairs.report
    if pairs.cache is not None:
        d[prefix + "cache_in"] = pairs.cache.view(np.uint8).reshape(-1, 16)
    if cache_out is not None:
        d[prefix + "cache_out"] = cache_out.view(np.uint8).reshape(-1, 16)
    for f in OUT_FIELDS:
        d[prefix + f] = getattr(out, f)


def unpack_case(z, prefix):
    g = lambda k: z[prefix + k] if (prefix + k) in z else None
    cache = g("cache_in")
    pairs = A.HostPairs(*(z[prefix + f] for f in PAIR_FIELDS), report=g("report"),
                        cache=None if cache is None else cache.reshape(-1).view(A.CACHE_DTYPE).copy())
    out = A.HostContacts(pairs.n, z[prefix + "normal_depth"].shape[0])
    for f in OUT_FIELDS:
        getattr(out, f)[...] = z[prefix + f]
    cache_out = g("cache_out")
    return (int(z[prefix + "algo"]), bool(int(z[prefix + "clip"])), pairs, out,
            None if cache_out is None else cache_out.reshape(-1).view(A.CACHE_DTYPE))


def case_prefixes(z):
    return sorted({k[: k.index("algo")] for k in z.files if k.endswith("algo")})


MANIFOLD_FIELDS = ("is_colliding", "nb_contacts", "normal_depth", "local1", "local2")


def manifold_groups(z):
    return sorted({k[: -len("_kept")] for k in z.files if k.endswith("_kept")})


def unpack_manifold(z, name):
    """(pairs, raw contacts, reduced contacts, kept table) of one group of
    np_manifold.npz; the pairs carry only the shape-1 poses."""
    rot1 = z[name + "_rot1"]
    n = len(rot1)
    zi = np.zeros(n, np.int32)
    pairs = A.HostPairs(zi, zi, z[name + "_pos1"], rot1, np.zeros((n, 4)), np.tile([0, 0, 0, 1.0], (n, 1)))
    mc = z[name + "_normal_depth"].shape[0]
    raw, red = A.HostContacts(n, mc), A.HostContacts(n, mc)
    for f in MANIFOLD_FIELDS:
        getattr(raw, f)[...] = z[name + "_" + f]
        getattr(red, f)[...] = z[name + "_red_" + f]
    return pairs, raw, red, z[name + "_kept"]
