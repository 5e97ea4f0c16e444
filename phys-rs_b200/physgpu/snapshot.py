"""Scene snapshots in the reference's save format (src/core/serialization.rs).

The reference saves a `SavedSimulation { entities: Vec<SavedEntity> }` with
`bincode::serialize_into` (bincode 1.3, default options) and loads it with
`bincode::deserialize_from` (src/render/surface.rs:853-928).  That encoding
is: little-endian fixed-width integers; a sequence as a u64 length then its
elements; a string as a u64 byte length then UTF-8; `Option` as a u8 tag
(0 = None, 1 = Some) then the value; a unit enum variant as its u32 index;
newtype structs as their inner value; glam's DVec3 / I64Vec3 as three
f64 / i64 with no length.  SavedEntity's fields, in declaration order
(serialization.rs:6-16):

    name: Option<EntityName(String)>      body_type: Option<BodyType>
    mass: Option<Mass(f64)>               radius: Option<BoundingRadius(f64)>
    local_pos: Option<LocalPosition(DVec3)>
    sector: Option<Sector(I64Vec3)>       velocity: Option<Velocity(DVec3)>
    temperature: Option<Temperature(f64)>

`load_world` turns a snapshot into the gravity path's World the way the
reference's loader spawns entities (surface.rs:905-920): entities without a
LocalPosition are not bodies; mass defaults to 1.0 (the loader's
`unwrap_or(1.0)`), sector and velocity to zero, Force and Acceleration start
at zero.
"""
import struct
from dataclasses import dataclass
from typing import List, Optional, Tuple

import numpy as np

# BodyType variants in declaration order (src/components/identifiers.rs:14-35)
BODY_TYPES = ("Star", "Planet", "Moon", "Asteroid", "Particle", "FluidParticle",
              "WhiteDwarf", "NeutronStar", "BlackHole")

Vec3 = Tuple[float, float, float]


@dataclass
class SavedEntity:
    """src/core/serialization.rs:6-16; every field optional."""
    name: Optional[str] = None
    body_type: Optional[str] = None
    mass: Optional[float] = None
    radius: Optional[float] = None
    local_pos: Optional[Vec3] = None
    sector: Optional[Tuple[int, int, int]] = None
    velocity: Optional[Vec3] = None
    temperature: Optional[float] = None


class SnapshotError(ValueError):
    pass


def encode(entities: List[SavedEntity]) -> bytes:
    """bincode 1.3 bytes of SavedSimulation { entities }."""
    out = [struct.pack("<Q", len(entities))]

    def opt(v, fmt):
        if v is None:
            out.append(b"\x00")
        else:
            out.append(b"\x01" + struct.pack(fmt, *v))

    for e in entities:
        if e.name is None:
            out.append(b"\x00")
        else:
            raw = e.name.encode("utf-8")
            out.append(b"\x01" + struct.pack("<Q", len(raw)) + raw)
        if e.body_type is None:
            out.append(b"\x00")
        else:
            if e.body_type not in BODY_TYPES:
                raise SnapshotError("unknown body type %r" % (e.body_type,))
            out.append(b"\x01" + struct.pack("<I", BODY_TYPES.index(e.body_type)))
        opt(None if e.mass is None else (e.mass,), "<d")
        opt(None if e.radius is None else (e.radius,), "<d")
        opt(e.local_pos, "<3d")
        opt(e.sector, "<3q")
        opt(e.velocity, "<3d")
        opt(None if e.temperature is None else (e.temperature,), "<d")
    return b"".join(out)


def decode(data: bytes) -> List[SavedEntity]:
    """SavedSimulation entities from bincode 1.3 bytes; raises SnapshotError
    on a truncated or malformed stream (bad tag, variant or UTF-8)."""
    mv = memoryview(data)
    pos = 0

    def take(fmt):
        nonlocal pos
        size = struct.calcsize(fmt)
        if pos + size > len(mv):
            raise SnapshotError("truncated snapshot at byte %d" % pos)
        v = struct.unpack_from(fmt, mv, pos)
        pos += size
        return v

    def tag():
        (t,) = take("<B")
        if t > 1:
            raise SnapshotError("invalid Option tag %d at byte %d" % (t, pos - 1))
        return t == 1

    (n,) = take("<Q")
    if n * 8 > len(mv) - pos:  # every entity takes at least its 8 Option tags
        raise SnapshotError("entity count %d exceeds the data" % n)
    ents = []
    for _ in range(n):
        e = SavedEntity()
        if tag():
            (ln,) = take("<Q")
            if pos + ln > len(mv):
                raise SnapshotError("truncated name at byte %d" % pos)
            try:
                e.name = bytes(mv[pos:pos + ln]).decode("utf-8")
            except UnicodeDecodeError as ex:
                raise SnapshotError("name is not UTF-8: %s" % ex) from None
            pos += ln
        if tag():
            (k,) = take("<I")
            if k >= len(BODY_TYPES):
                raise SnapshotError("invalid BodyType variant %d" % k)
            e.body_type = BODY_TYPES[k]
        if tag():
            (e.mass,) = take("<d")
        if tag():
            (e.radius,) = take("<d")
        if tag():
            e.local_pos = take("<3d")
        if tag():
            e.sector = take("<3q")
        if tag():
            e.velocity = take("<3d")
        if tag():
            (e.temperature,) = take("<d")
        ents.append(e)
    if pos != len(mv):
        raise SnapshotError("%d trailing bytes after the snapshot" % (len(mv) - pos))
    return ents


def save(entities: List[SavedEntity], path) -> None:
    with open(path, "wb") as f:
        f.write(encode(entities))


def load(path) -> List[SavedEntity]:
    with open(path, "rb") as f:
        return decode(f.read())


def world_entities(world, names=None, body_types=None, radii=None, temperatures=None):
    """SavedEntity list for the bodies of a World (the QuickSave query,
    surface.rs:853-877); the optional per-body lists fill the fields the
    gravity path does not carry."""
    ents = []
    for i in range(len(world)):
        ents.append(SavedEntity(
            name=None if names is None else names[i],
            body_type=None if body_types is None else body_types[i],
            mass=float(world.mass[i]),
            radius=None if radii is None else float(radii[i]),
            local_pos=tuple(float(v) for v in world.local[i]),
            sector=tuple(int(v) for v in world.sector[i]),
            velocity=tuple(float(v) for v in world.velocity[i]),
            temperature=None if temperatures is None else float(temperatures[i])))
    return ents


def load_world(path_or_entities):
    """World of the snapshot's bodies, spawned as the reference's QuickLoad
    does (surface.rs:905-920).  Returns (world, entity_index): entity_index[k]
    is the snapshot entity of body k."""
    from . import World
    ents = load(path_or_entities) if not isinstance(path_or_entities, list) else path_or_entities
    idx = [k for k, e in enumerate(ents) if e.local_pos is not None]
    bodies = [ents[k] for k in idx]
    n = len(bodies)
    w = World()
    w.mass = np.array([1.0 if e.mass is None else e.mass for e in bodies], dtype=np.float64)
    w.local = np.array([e.local_pos for e in bodies], dtype=np.float64).reshape(n, 3)
    w.sector = np.array([(0, 0, 0) if e.sector is None else e.sector for e in bodies],
                        dtype=np.int64).reshape(n, 3)
    w.velocity = np.array([(0.0, 0.0, 0.0) if e.velocity is None else e.velocity
                           for e in bodies], dtype=np.float64).reshape(n, 3)
    w.force = np.zeros((n, 3))
    w.acceleration = np.zeros((n, 3))
    w.prev_acceleration = np.zeros((n, 3))
    return w, np.array(idx, dtype=np.int64)
