"""Saving and loading network state.

Files have the reference's layout and formats (ANNarchy/core/IO.py:340-617,
Population.py:1000-1115, Projection.py:1731-1950), so a state saved by one
simulator can be loaded by the other: a dict with "time_step", "net_id",
"obj_names" and one entry per population (name, geometry, size, attribute
lists, every attribute: local ones reshaped to the geometry) and per
projection (name, pre, post, target, post_ranks, pre_ranks per dendrite,
delays, every synaptic attribute per dendrite). ".npz" uses
np.savez_compressed, ".gz" a gzip'ed pickle, ".mat" scipy.io.savemat (not
loadable), anything else a plain pickle. Attribute values are read from and
written to the device arrays through the C ABI.
"""
from __future__ import annotations

import gzip
import os
import pickle

import numpy as np
import scipy.sparse as sp


def save_data(filename: str, data: dict):
    path = os.path.dirname(filename)
    if path and not os.path.isdir(path):
        os.makedirs(path)
    ext = os.path.splitext(filename)[1]
    if ext == ".mat":
        import scipy.io as sio
        sio.savemat(filename, data)
    elif ext == ".gz":
        with gzip.open(filename, mode="wb") as f:
            pickle.dump(data, f, protocol=pickle.HIGHEST_PROTOCOL)
    elif ext == ".npz":
        np.savez_compressed(filename, allow_pickle=True, **data)
    else:
        with open(filename, mode="wb") as f:
            pickle.dump(data, f, protocol=pickle.HIGHEST_PROTOCOL)


def load_data(filename: str, pickle_encoding: str | None = None) -> dict:
    ext = os.path.splitext(filename)[1]
    kw = {} if pickle_encoding is None else {"encoding": pickle_encoding}
    if ext == ".mat":
        raise ValueError("Matlab files can not be loaded")
    if ext == ".gz":
        with gzip.open(filename, mode="rb") as f:
            return pickle.load(f, **kw)
    if ext == ".npz":
        data = np.load(filename, allow_pickle=True, **kw)
        out = {}
        for key in data.files:
            v = data[key]
            out[key] = v.item(0) if v.dtype == np.dtype("O") and v.ndim == 0 else v
        return out
    with open(filename, mode="rb") as f:
        return pickle.load(f, **kw)


# -------------------------------------------------------------------- populations
def population_data(pop) -> dict:
    desc = {"name": pop.name, "geometry": pop.geometry, "size": pop.size}
    d = pop.desc
    desc["attributes"] = list(d["attributes"])
    desc["parameters"] = [p["name"] for p in d["parameters"]]
    desc["variables"] = [v["name"] for v in d["variables"]]
    for var in d["parameters"] + d["variables"]:
        name = var["name"]
        if name not in pop._host:
            continue
        value = pop.get(name)
        if var["locality"] == "local":
            dtype = bool if var.get("ctype") == "bool" else (int if var.get("ctype") == "int" else float)
            desc[name] = np.asarray(value, dtype=dtype).reshape(pop.geometry)
        else:
            desc[name] = value
    return desc


def load_population_data(pop, desc: dict):
    if "attributes" not in desc:
        raise ValueError("the file holds no population attributes")
    for name in desc["attributes"]:
        if name not in pop._host or name not in desc:
            continue
        value = desc[name]
        if isinstance(value, np.ndarray):
            value = value.reshape(-1) if pop._locality.get(name) == "local" else value.reshape(()).item()
        pop.set({name: value})


# -------------------------------------------------------------------- projections
def _pre_ranks(proj) -> list:
    m = proj._csr
    lengths = np.diff(m.indptr)
    rows = np.nonzero(lengths > 0)[0]
    return [proj.pre_ranks[m.indices[m.indptr[r]:m.indptr[r + 1]]].tolist() for r in rows]


def _per_dendrite(values: list):
    """Per-dendrite values as the reference stores them: a 2-D array when
    every dendrite has the same size, else an object array of lists."""
    ragged = len({len(v) for v in values}) > 1
    if ragged:
        out = np.empty(len(values), dtype=object)
        for i, v in enumerate(values):
            out[i] = np.asarray(v).tolist()
        return out
    return np.array([np.asarray(v) for v in values])


def projection_data(proj) -> dict:
    if getattr(proj, "_device_conn", None):
        raise NotImplementedError("projections generated on the device are not saved by this backend")
    desc = {"name": proj.name, "pre": proj.pre_pop.name, "post": proj.post_pop.name,
            "target": proj.target, "post_ranks": proj.post_ranks}
    d = proj.desc
    desc["attributes"] = [p["name"] for p in d["parameters"] + d["variables"]]
    if "w" not in desc["attributes"]:
        desc["attributes"].append("w")
    desc["parameters"] = [p["name"] for p in d["parameters"]]
    desc["variables"] = [v["name"] for v in d["variables"]]
    desc["delays"] = proj.delay
    desc["pre_ranks"] = _per_dendrite(_pre_ranks(proj))
    glob = {p["name"] for p in d["parameters"] + d["variables"] if p["locality"] == "global"}
    for name in desc["attributes"]:
        if name in glob:
            desc[name] = proj.get(name)
        elif name in proj._host_semi:                     # one value per dendrite
            desc[name] = np.asarray(proj.get(name), dtype=np.float64)
        elif name in proj._attr_names():
            desc[name] = _per_dendrite([np.asarray(v) for v in proj.get(name)])
    return desc


def load_projection_data(proj, desc: dict):
    """Before compile(): the connectivity, weights and delays of the file
    become the projection's (like a connector). After compile(): the
    connectivity must be the same; the synaptic attributes and the delays
    are loaded."""
    post_ranks = [int(r) for r in desc["post_ranks"]]
    pre_ranks = [list(map(int, r)) for r in desc["pre_ranks"]]
    w = [np.atleast_1d(np.asarray(v, dtype=np.float64)) for v in desc["w"]]
    compiled = proj.net is not None and proj.net._compiled
    if not compiled:
        pos_post = {int(r): i for i, r in enumerate(proj.post_ranks_view)}
        pos_pre = {int(r): i for i, r in enumerate(proj.pre_ranks)}
        rows = np.concatenate([np.full(len(p), pos_post[r]) for r, p in zip(post_ranks, pre_ranks)])
        cols = np.concatenate([[pos_pre[c] for c in p] for p in pre_ranks]).astype(np.int64)
        m = sp.csr_matrix((np.concatenate(w), (rows, cols)),
                          shape=(len(proj.post_ranks_view), len(proj.pre_ranks)))
        delays = desc.get("delays", 0.0)
        if isinstance(delays, (list, np.ndarray)) and np.ndim(delays) > 0:
            dm = sp.csr_matrix((np.concatenate([np.atleast_1d(np.asarray(v, dtype=np.float64))
                                                for v in delays]), (rows, cols)), shape=m.shape)
            proj._store(m, "Load", None, None, dm)
        else:
            proj._store(m, "Load", None, float(delays))
    else:
        if post_ranks != list(proj.post_ranks) or pre_ranks != _pre_ranks(proj):
            raise ValueError(f"{proj.name}: the file's connectivity differs from the compiled one; "
                             "load it before compile()")
        proj.set({"w": w})
        if "delays" in desc:
            proj.delay = desc["delays"]
    d = proj.desc
    for v in d["parameters"] + d["variables"]:
        name = v["name"]
        if name == "w" or name not in desc:
            continue
        if v["locality"] == "global":
            proj.set({name: float(np.asarray(desc[name]).reshape(-1)[0])})
        elif name in proj._host_semi:
            proj.set({name: np.asarray(desc[name], dtype=np.float64).reshape(-1)})
        elif name in proj._attr_names():
            proj.set({name: [np.atleast_1d(np.asarray(x, dtype=np.float64)) for x in desc[name]]})


# -------------------------------------------------------------------- networks
def network_description(net, populations=True, projections=True) -> dict:
    desc = {"time_step": net.current_step, "net_id": net.id}
    pops, projs = [], []
    if populations:
        for pop in net.populations:
            desc[pop.name] = population_data(pop)
            pops.append(pop.name)
    if projections:
        for proj in net.projections:
            if getattr(proj, "_device_conn", None):
                continue
            desc[proj.name] = projection_data(proj)
            projs.append(proj.name)
    desc["obj_names"] = {"populations": pops, "projections": projs}
    return desc


def load_network(net, desc: dict, populations=True, projections=True):
    if "time_step" in desc and net._compiled:
        net.set_current_step(int(np.asarray(desc["time_step"])))
    if populations:
        for pop in net.populations:
            if pop.name in desc:
                load_population_data(pop, desc[pop.name])
    if projections:
        for proj in net.projections:
            if proj.name in desc:
                load_projection_data(proj, desc[proj.name])
