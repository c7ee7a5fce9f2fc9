"""Huffman-compressed grid volumes (pine's `.compressed` format, fileio.cpp:204-249 and
util/huffman.h): a file written here by a restatement of pine's encoder reads back to the
same densities, damaged files are rejected, and pine's shipped `wdas_cloud.compressed`
decodes completely when the reference tree is present on this machine."""
import heapq
import os
import struct

import numpy as np
import pytest

import oracle


def _codes(values):
    """Prefix-free codes (Huffman) as pine stores them: the path bits, least significant
    first, under a leading 1."""
    uniq, counts = np.unique(values, return_counts=True)
    if len(uniq) == 1:
        return {int(uniq[0]): 1}
    heap = [(int(c), i, [int(v)]) for i, (v, c) in enumerate(zip(uniq, counts))]
    heapq.heapify(heap)
    path = {int(v): (0, 0) for v in uniq}  # value -> (bits, length)
    k = len(heap)
    while len(heap) > 1:
        c0, _, g0 = heapq.heappop(heap)
        c1, _, g1 = heapq.heappop(heap)
        for bit, g in ((0, g0), (1, g1)):
            for v in g:
                b, n = path[v]
                path[v] = ((b << 1) | bit, n + 1)
        heapq.heappush(heap, (c0 + c1, k, g0 + g1))
        k += 1
    # Each merge shifts the paths left and adds its bit at the bottom (huffman.h:71-72), so
    # the bit nearest the root is the least significant one, the first the decoder reads.
    return {v: (1 << n) | b for v, (b, n) in path.items()}


def write_compressed(path, density, size):
    # CompressVolume's quantisation (fileio.cpp:204-229): min(d, 32) * 65535 / 32 in float,
    # truncated to 16 bits; LoadCompressedVolume divides by float(65535 / 32) = 2047.
    vals = np.minimum(density, np.float32(32.0)).astype(np.float32)
    q = (vals * np.float32(65535) / np.float32(32)).astype(np.uint16)
    codes = _codes(q)
    bits = []
    for v in q.ravel():
        c = codes[int(v)]
        h = c.bit_length() - 1
        bits.extend((c >> j) & 1 for j in range(h))
    nbits = len(bits)
    data = np.packbits(np.array(bits + [0] * (-nbits % 8), np.uint8), bitorder="little")
    tree = bytearray(56)
    struct.pack_into("<Q", tree, 24, len(codes))
    for v, c in codes.items():
        tree += struct.pack("<HI", v, c)
    enc = struct.pack("<QQQ", 0x1000, 0x1000 + len(data), 0x1000 + len(data))
    enc += data.tobytes() + struct.pack("<IQ", nbits, q.size)
    with open(path, "wb") as f:
        f.write(struct.pack("<3iQQ", *size, len(tree), len(enc)) + bytes(tree) + enc)
    return q.astype(np.float32) / 2047.0


def _scene(tmp_path, volfile):
    p = tmp_path / "c.txt"
    p.write_text("Integrator: Path{\n maxDepth: 8\n sampler: Uniform{\n samplesPerPixel: 4\n }\n}\n"
                 "Camera: ThinLen{\n film{\n size: 32 24\n filter: Box{\n radius: 0.5\n }\n }\n"
                 " from: -4 0.5 0\n to: 0.5 0.5 0.5\n fov: 0.5\n medium: cloud\n}\n"
                 "Light: Environment{\n environment: Sky{\n sunDirection: -1 6 1\n sunColor: 1\n }\n}\n"
                 f"Medium cloud: Grid{{\n file: {volfile}\n sigma_a: 1\n sigma_s: 20\n g: 0.0\n"
                 " position: 0 0 0\n scale: 1.0\n}\n")
    return str(p)


def _density(desc):
    m = desc.media[0]
    n = m.size[0] * m.size[1] * m.size[2]
    return np.ctypeslib.as_array(m.density, shape=(n,)).copy(), tuple(m.size)


def test_round_trip(pglib, tmp_path):
    import pine_b200 as pb
    rng = np.random.default_rng(3)
    size = (13, 7, 11)
    dens = np.where(rng.uniform(size=size[::-1]) < 0.6, 0.0, rng.gamma(2.0, 3.0, size[::-1]))
    want = write_compressed(tmp_path / "v.compressed", dens.astype(np.float32), size)
    ps = pb.ParsedScene(_scene(tmp_path, "v.compressed"))
    got, gsize = _density(ps.desc)
    ps.close()
    assert gsize == size
    np.testing.assert_array_equal(got, want.ravel())


def test_single_value_volume(pglib, tmp_path):
    import pine_b200 as pb
    want = write_compressed(tmp_path / "v.compressed", np.full((3, 2, 2), 1.5, np.float32), (2, 2, 3))
    ps = pb.ParsedScene(_scene(tmp_path, "v.compressed"))
    got, _ = _density(ps.desc)
    ps.close()
    np.testing.assert_array_equal(got, want.ravel())


@pytest.mark.parametrize("damage", ["truncate", "count", "bits", "wrapped_vector",
                                    "wrapped_tree"])
def test_damaged_files_are_rejected(pglib, tmp_path, damage):
    import pine_b200 as pb
    rng = np.random.default_rng(4)
    write_compressed(tmp_path / "v.compressed", rng.uniform(0, 5, (4, 4, 4)).astype(np.float32),
                     (4, 4, 4))
    raw = bytearray((tmp_path / "v.compressed").read_bytes())
    tree_bytes = struct.unpack_from("<Q", raw, 12)[0]
    if damage == "truncate":
        raw = raw[:-5]
    elif damage == "count":
        raw[-8:] = struct.pack("<Q", 65)
    elif damage == "bits":
        nb = struct.unpack_from("<I", raw, len(raw) - 12)[0]
        struct.pack_into("<I", raw, len(raw) - 12, nb - 3)
    elif damage == "wrapped_vector":
        # A 30-byte encoded section whose vector claims 2^64 - 6 bytes: 24 + that + 12
        # wraps around to 30.
        enc = 28 + tree_bytes
        raw = raw[:enc + 30]
        struct.pack_into("<Q", raw, 20, 30)
        struct.pack_into("<QQ", raw, enc, 0, (1 << 64) - 6)
    else:
        # A tree size that makes the three section sizes wrap around to the file size.
        enc_bytes = struct.unpack_from("<Q", raw, 20)[0]
        struct.pack_into("<Q", raw, 12, (1 << 64) - 8)
        struct.pack_into("<Q", raw, 20, (len(raw) - 28 + 8 + enc_bytes) - enc_bytes)
    (tmp_path / "v.compressed").write_bytes(bytes(raw))
    with pytest.raises(pb.PgError) as e:
        pb.ParsedScene(_scene(tmp_path, "v.compressed"))
    assert e.value.status == 7  # PG_ERR_PARSE


SHIPPED = os.path.join(oracle.REFERENCE_SRC, "scenes", "wdas_cloud.compressed")


@pytest.mark.skipif(not os.path.exists(SHIPPED), reason="the reference tree is not present")
def test_shipped_cloud_decodes(pglib, tmp_path):
    """pine's own cloud scene data: every voxel of the 250 x 170 x 307 grid decodes from
    exactly the stored bit count (pine's reader for it is commented out)."""
    import pine_b200 as pb
    os.symlink(SHIPPED, tmp_path / "wdas_cloud.compressed")
    ps = pb.ParsedScene(_scene(tmp_path, "wdas_cloud.compressed"))
    dens, size = _density(ps.desc)
    ps.close()
    assert size == (250, 170, 307)
    assert dens.min() >= 0.0 and dens.max() <= 32.0 + 1e-3
    assert 0.05 < np.mean(dens > 0) < 0.95
