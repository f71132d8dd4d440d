"""The editor's emitter graph -> simulation sources.

Restates src/store/node-store/sourceGraph.ts:103-132 (resolveEmitterSources)
and the props mapping of src/store/node-store/nodeStore.ts:49-109
(emitterPropsToSource), so a host without the editor can feed
fx_sim_update_sources (through packEmitterSources) from a saved graph:
- an emitter is a source when a directed path leads from it to the
  'combustion' node;
- a velocity or igniter emitter linked (either way, through emitter-to-emitter
  edges) to a scalar or burst emitter takes the position of the nearest such
  emitter (breadth-first over the links); an igniter also takes the larger of
  the two radii.
Emitter ids start with 'emitter-'.
"""
from __future__ import annotations

import dataclasses
from collections import deque
from typing import Any, Dict, List, Mapping, Optional, Sequence

from .emitters import BurstEmitter, IgniterEmitter, ScalarEmitter, VelocityEmitter


def _pos(p: Mapping[str, Any]):
    return (float(p["positionX"]), float(p["positionY"]), float(p["positionZ"]))


def emitter_props_to_source(props: Mapping[str, Any]):
    """EmitterNodeProps -> the emitter dataclass of its kind."""
    kind = props["kind"]
    common = dict(position=_pos(props), radius=props["radius"], startTime=props["startTime"], duration=props["duration"])
    if kind == "scalar":
        return ScalarEmitter(**common, densityRate=props["densityRate"], heatRate=props["heatRate"], fuelRate=props["fuelRate"],
                             noiseScale=props["noiseScale"], noiseMix=props["noiseMix"], seed=props["seed"])
    if kind == "velocity":
        return VelocityEmitter(**common, mode=props["mode"], speed=props["speed"],
                               direction=(props["directionX"], props["directionY"], props["directionZ"]), falloff=props["falloff"],
                               seed=props["seed"], tightness=props.get("tightness") if props.get("tightness") is not None else 0.0)
    if kind == "burst":
        return BurstEmitter(**common, densityAmount=props["densityAmount"], heatAmount=props["heatAmount"], fuelAmount=props["fuelAmount"],
                            reactionAmount=props["reactionAmount"], expansionSpeed=props["expansionSpeed"], liftSpeed=props["liftSpeed"],
                            turbulenceSpeed=props["turbulenceSpeed"], falloff=props["falloff"], noiseScale=props["noiseScale"],
                            noiseMix=props["noiseMix"], seed=props["seed"])
    return IgniterEmitter(**common, intensity=props["intensity"], seed=props["seed"])


def _is_emitter(node_id: str) -> bool:
    return node_id.startswith("emitter-")


def _is_material(emitter: Mapping[str, Any]) -> bool:
    return emitter["props"]["kind"] in ("scalar", "burst")


def resolve_emitter_sources(emitters: Sequence[Mapping[str, Any]], edges: Sequence[Mapping[str, str]]) -> List[Any]:
    """emitters: [{"id", "label", "props"}], edges: [{"source", "target"}] ->
    the sources in emitter order."""
    outgoing: Dict[str, List[str]] = {}
    links: Dict[str, List[str]] = {}
    for e in edges:
        outgoing.setdefault(e["source"], []).append(e["target"])
        if _is_emitter(e["source"]) and _is_emitter(e["target"]):
            links.setdefault(e["source"], []).append(e["target"])
            links.setdefault(e["target"], []).append(e["source"])
    by_id = {e["id"]: e for e in emitters}

    def reaches_combustion(start: str) -> bool:
        seen, stack = set(), [start]
        while stack:
            cur = stack.pop()
            if cur in seen:
                continue
            if cur == "combustion":
                return True
            seen.add(cur)
            stack.extend(outgoing.get(cur, []))
        return False

    def nearest_material(start: str) -> Optional[Mapping[str, Any]]:
        first = by_id.get(start)
        if first is None or _is_material(first):
            return None
        seen, queue = set(), deque([start])
        while queue:
            cur = queue.popleft()
            if cur in seen:
                continue
            seen.add(cur)
            em = by_id.get(cur)
            if em is not None and _is_material(em):
                return em
            queue.extend(links.get(cur, []))
        return None

    out = []
    for em in emitters:
        if not reaches_combustion(em["id"]):
            continue
        src = emitter_props_to_source(em["props"])
        anchor = nearest_material(em["id"])
        if anchor is not None:
            a = emitter_props_to_source(anchor["props"])
            src = dataclasses.replace(src, position=tuple(a.position))
            if src.kind == "igniter":
                src = dataclasses.replace(src, radius=max(src.radius, a.radius))
        out.append(src)
    return out
