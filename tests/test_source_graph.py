"""resolve_emitter_sources (sourceGraph.ts:103-132) and the packing it feeds."""
from fenix_b200 import packEmitterSources
from fenix_b200.source_graph import emitter_props_to_source, resolve_emitter_sources


def scalar(x, r=0.05):
    return {"kind": "scalar", "positionX": x, "positionY": 0.1, "positionZ": 0.5, "radius": r, "startTime": 0.0, "duration": 10.0,
            "densityRate": 1.0, "heatRate": 2.0, "fuelRate": 3.0, "noiseScale": 4.0, "noiseMix": 0.5, "seed": 7.0}


def velocity(x):
    return {"kind": "velocity", "positionX": x, "positionY": 0.9, "positionZ": 0.9, "radius": 0.2, "startTime": 0.0, "duration": 10.0,
            "mode": "directional", "speed": 5.0, "directionX": 0.0, "directionY": 1.0, "directionZ": 0.0, "falloff": 0.4, "seed": 3.0}


def igniter(x, r):
    return {"kind": "igniter", "positionX": x, "positionY": 0.5, "positionZ": 0.5, "radius": r, "startTime": 0.0, "duration": 1.0,
            "intensity": 0.8, "seed": 9.0}


def em(i, props):
    return {"id": f"emitter-{i}", "label": str(i), "props": props}


def test_only_emitters_reaching_combustion_are_sources():
    emitters = [em(0, scalar(0.2)), em(1, scalar(0.4)), em(2, velocity(0.6))]
    edges = [{"source": "emitter-0", "target": "combustion"}, {"source": "emitter-2", "target": "mixer"},
             {"source": "mixer", "target": "combustion"}]
    out = resolve_emitter_sources(emitters, edges)
    assert [s.kind for s in out] == ["scalar", "velocity"]
    assert out[1].position == (0.6, 0.9, 0.9) and out[1].tightness == 0.0  # not linked to a material emitter


def test_channels_inherit_the_nearest_material_source():
    emitters = [em(0, scalar(0.2, r=0.05)), em(1, velocity(0.9)), em(2, igniter(0.7, r=0.01)), em(3, scalar(0.6, r=0.3)),
                em(4, igniter(0.1, r=0.5))]
    edges = [{"source": f"emitter-{i}", "target": "combustion"} for i in range(5)]
    edges += [{"source": "emitter-1", "target": "emitter-0"},          # velocity -> scalar 0
              {"source": "emitter-3", "target": "emitter-2"},          # scalar 3 -> igniter (undirected link)
              {"source": "emitter-4", "target": "emitter-1"}]          # igniter 4 -> velocity -> scalar 0 (two hops)
    out = resolve_emitter_sources(emitters, edges)
    assert out[1].position == (0.2, 0.1, 0.5)
    assert out[2].position == (0.6, 0.1, 0.5) and out[2].radius == 0.3
    assert out[4].position == (0.2, 0.1, 0.5) and out[4].radius == 0.5
    assert out[0].position == (0.2, 0.1, 0.5)  # material sources keep their own
    packed = packEmitterSources(out)
    assert packed.shape == (5 * 32,)


def test_props_mapping_and_cycles():
    s = emitter_props_to_source(scalar(0.3))
    assert (s.kind, s.densityRate, s.heatRate, s.fuelRate) == ("scalar", 1.0, 2.0, 3.0)
    emitters = [em(0, velocity(0.5)), em(1, velocity(0.6))]
    edges = [{"source": "emitter-0", "target": "emitter-1"}, {"source": "emitter-1", "target": "emitter-0"},
             {"source": "emitter-1", "target": "combustion"}]
    out = resolve_emitter_sources(emitters, edges)  # the cycle terminates; no material anchor
    assert [o.position for o in out] == [(0.5, 0.9, 0.9), (0.6, 0.9, 0.9)]
