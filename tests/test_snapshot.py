"""Scene snapshots in the reference's save format (serialization.rs, bincode
1.3 default options).  Parity is unpinned: the reference tree holds no save
file and cargo is absent, so the byte layout below is built by hand from
bincode 1.3's published encoding and serde's field order, and the product's
encoder and decoder are checked against it, against each other, and against
malformed input."""
import struct

import numpy as np
import pytest

import physgpu
from physgpu import snapshot as snap


def hand_bytes():
    """Two entities written field by field: a fully populated star and a
    body with only a position."""
    b = struct.pack("<Q", 2)
    name = "Sun".encode()
    b += b"\x01" + struct.pack("<Q", len(name)) + name         # name
    b += b"\x01" + struct.pack("<I", 0)                          # BodyType::Star
    b += b"\x01" + struct.pack("<d", 1.989e30)                   # mass
    b += b"\x01" + struct.pack("<d", 6.96e8)                     # radius
    b += b"\x01" + struct.pack("<3d", 1.0, -2.0, 3.5)            # local_pos
    b += b"\x01" + struct.pack("<3q", -1, 0, 7)                  # sector
    b += b"\x01" + struct.pack("<3d", 0.0, 2.9e4, -1.0)          # velocity
    b += b"\x01" + struct.pack("<d", 5772.0)                     # temperature
    b += b"\x00" * 4 + b"\x01" + struct.pack("<3d", 9.0, 8.0, 7.0) + b"\x00" * 3
    return b


def test_decode_hand_built_layout():
    ents = snap.decode(hand_bytes())
    assert len(ents) == 2
    s, p = ents
    assert (s.name, s.body_type, s.mass, s.radius) == ("Sun", "Star", 1.989e30, 6.96e8)
    assert s.local_pos == (1.0, -2.0, 3.5) and s.sector == (-1, 0, 7)
    assert s.velocity == (0.0, 2.9e4, -1.0) and s.temperature == 5772.0
    assert p == snap.SavedEntity(local_pos=(9.0, 8.0, 7.0))


def test_encode_is_the_same_layout_and_round_trips():
    ents = snap.decode(hand_bytes())
    assert snap.encode(ents) == hand_bytes()
    rng = np.random.default_rng(0)
    many = []
    for i in range(200):
        many.append(snap.SavedEntity(
            name=None if i % 3 == 0 else "body-%d-é" % i,
            body_type=None if i % 5 == 0 else snap.BODY_TYPES[i % 9],
            mass=None if i % 7 == 0 else float(rng.lognormal()),
            radius=None if i % 2 else float(rng.random()),
            local_pos=None if i % 11 == 0 else tuple(rng.normal(size=3)),
            sector=None if i % 4 else tuple(int(v) for v in rng.integers(-9, 9, 3)),
            velocity=None if i % 6 == 0 else tuple(rng.normal(size=3)),
            temperature=None if i % 8 else float(rng.random() * 1e4)))
    assert snap.decode(snap.encode(many)) == many
    assert snap.encode([]) == struct.pack("<Q", 0)


def test_malformed_streams_are_rejected():
    good = hand_bytes()
    for cut in (3, 9, 20, len(good) - 1):
        with pytest.raises(snap.SnapshotError):
            snap.decode(good[:cut])
    with pytest.raises(snap.SnapshotError):
        snap.decode(good + b"\x00")  # trailing bytes
    bad_tag = bytearray(good)
    bad_tag[8] = 2
    with pytest.raises(snap.SnapshotError):
        snap.decode(bytes(bad_tag))
    bad_variant = snap.encode([snap.SavedEntity(body_type="Moon")])
    bad_variant = bad_variant[:10] + struct.pack("<I", 9) + bad_variant[14:]
    with pytest.raises(snap.SnapshotError):
        snap.decode(bad_variant)
    with pytest.raises(snap.SnapshotError):
        snap.decode(struct.pack("<Q", 1 << 40))
    with pytest.raises(snap.SnapshotError):
        snap.encode([snap.SavedEntity(body_type="Comet")])


def test_world_round_trip_and_loader_defaults(tmp_path):
    """QuickSave of a World and QuickLoad back (surface.rs:853-920): bodies
    only for entities with a LocalPosition, mass 1.0 when absent, sector and
    velocity zero when absent."""
    w = physgpu.World()
    w.spawn(2.0, [1.0, 2.0, 3.0], sector=[1, -2, 3], velocity=[0.5, 0.0, -0.5])
    w.spawn(3.0, [-1.0, 0.0, 4.0])
    path = tmp_path / "quicksave.bin"
    snap.save(snap.world_entities(w, names=["a", "b"], body_types=["Planet", "Moon"]), path)
    w2, idx = snap.load_world(path)
    assert list(idx) == [0, 1]
    for f in ("mass", "local", "sector", "velocity"):
        assert np.array_equal(getattr(w2, f), getattr(w, f)), f
    assert not w2.force.any() and not w2.acceleration.any()
    ents = [snap.SavedEntity(name="ghost"), snap.SavedEntity(local_pos=(1.0, 1.0, 1.0))]
    w3, idx3 = snap.load_world(ents)
    assert list(idx3) == [1] and w3.mass[0] == 1.0 and not w3.sector.any()
    assert not w3.velocity.any()
