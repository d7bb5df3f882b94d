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
