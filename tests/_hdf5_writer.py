"""Minimal HDF5 writer for test fixtures (test infrastructure only).

Writes the structures the library's HDF5 reader parses, laid out as the
HDF5 file-format specification describes them:
  - superblock version 0 with version 1 object headers and symbol-table groups
    (version 1 B-tree, symbol-table nodes, local heap), the layout libhdf5 1.8
    writes by default and in which EMAN stores its images;
  - superblock version 2 with version 2 ("OHDR") object headers and compact
    link messages (new-style groups).
Datasets are contiguous, compact or chunked (version 1 B-tree chunk index,
optional shuffle + deflate filters); attributes are scalars, 1D arrays or
fixed-length strings.  Checksums of version 2 structures are written as zero
(the reader does not verify them).  The node capacities are parameters so that
small groups already need several symbol-table nodes and B-tree levels.
"""
import struct
import zlib

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF
SIG = b"\x89HDF\r\n\x1a\n"


def _pad8(b):
    return b + b"\0" * (-len(b) % 8)


def _dtype_msg(dt):
    dt = np.dtype(dt)
    if dt.kind == "S":
        return bytes([0x13, 0, 0, 0]) + struct.pack("<I", dt.itemsize)
    big = 1 if dt.byteorder == ">" else 0
    if dt.kind in "iu":
        bits = big | (8 if dt.kind == "i" else 0)
        return bytes([0x10, bits, 0, 0]) + struct.pack("<IHH", dt.itemsize, 0, 8 * dt.itemsize)
    if dt.kind == "f":
        if dt.itemsize == 4:
            props = struct.pack("<HHBBBBI", 0, 32, 23, 8, 0, 23, 127)
            sign = 31
        else:
            props = struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)
            sign = 63
        return bytes([0x11, big | 0x20, sign, 0]) + struct.pack("<I", dt.itemsize) + props
    raise ValueError(dt)


def _space_msg(shape):
    return struct.pack("<BBBB4x", 1, len(shape), 0, 0) + b"".join(struct.pack("<Q", d) for d in shape)


class ClaimedShape:
    """An attribute whose dataspace claims `shape` while only `data` is
    stored (a corrupt file: the claimed size need not fit the message)."""

    def __init__(self, dtype, shape, data):
        self.dtype, self.shape, self.data = np.dtype(dtype), tuple(shape), bytes(data)


class Node:
    """A group (children by name) or a dataset, with attributes."""

    def __init__(self, data=None, chunks=None, filters=(), compact=False):
        self.children = {}
        self.attrs = {}
        self.data = data
        self.chunks = chunks
        self.filters = filters
        self.compact = compact

    def group(self, path):
        node = self
        for part in [p for p in path.split("/") if p]:
            node = node.children.setdefault(part, Node())
        return node

    def dataset(self, path, data, **kw):
        parts = [p for p in path.split("/") if p]
        parent = self.group("/".join(parts[:-1]))
        node = Node(np.asarray(data), **kw)
        parent.children[parts[-1]] = node
        return node


class Writer:
    def __init__(self, superblock=0, userblock=0, snod_capacity=8, btree_capacity=32, dense_links=False,
                 header_messages=None):
        self.sb = superblock
        self.userblock = userblock
        self.snod_cap = snod_capacity
        self.bt_cap = btree_capacity
        self.dense_links = dense_links
        # at most this many messages per header block; the rest go to chained
        # continuation blocks (as libhdf5 does when attributes keep being added)
        self.per_block = header_messages
        self.buf = bytearray()

    def _alloc(self, b):
        b = _pad8(bytes(b))
        addr = len(self.buf)
        self.buf += b
        return addr

    # -- object headers -------------------------------------------------
    def _msgs(self, msgs):
        if self.sb >= 2:
            return b"".join(struct.pack("<BHB", t, len(d), 0) + d for t, d in msgs)
        return b"".join(struct.pack("<HHB3x", t, len(_pad8(d)), 0) + _pad8(d) for t, d in msgs)

    def _header(self, msgs):
        n_all = len(msgs)
        k = self.per_block
        if k and len(msgs) > k:
            # chain: the last block first, each earlier block ending with a
            # continuation message (address, length) to the next
            blocks = [msgs[i:i + k] for i in range(0, len(msgs), k)]
            nxt = None
            for blk in reversed(blocks[1:]):
                blk = list(blk) + ([nxt] if nxt else [])
                body = self._msgs(blk)
                raw = (b"OCHK" + body + b"\0" * 4) if self.sb >= 2 else body
                addr = self._alloc(raw)
                nxt = (0x10, struct.pack("<QQ", addr, len(raw)))
                n_all += 1
            msgs = list(blocks[0]) + [nxt]
        body = self._msgs(msgs)
        if self.sb >= 2:
            return self._alloc(b"OHDR" + struct.pack("<BBI", 2, 2, len(body)) + body + b"\0" * 4)
        return self._alloc(struct.pack("<BBHII4x", 1, 0, n_all, 1, len(body)) + body)

    def _attr_msgs(self, attrs):
        out = []
        for name, val in attrs.items():
            if isinstance(val, ClaimedShape):
                dt, shape, data = _dtype_msg(val.dtype), val.shape, val.data
            elif isinstance(val, str):
                raw = val.encode() + b"\0"
                dt, shape, data = _dtype_msg("S%d" % len(raw)), (), raw
            else:
                a = np.asarray(val)
                dt, shape, data = _dtype_msg(a.dtype), a.shape, a.tobytes()
            nm = name.encode() + b"\0"
            sp = _space_msg(shape)
            if self.sb >= 2:
                body = struct.pack("<BBHHH", 2, 0, len(nm), len(dt), len(sp)) + nm + dt + sp + data
            else:
                body = (struct.pack("<BBHHH", 1, 0, len(nm), len(dt), len(sp)) + _pad8(nm) + _pad8(dt)
                        + _pad8(sp) + data)
            out.append((0x0C, body))
        return out

    # -- datasets ---------------------------------------------------------
    def _dataset(self, node):
        a = node.data
        msgs = [(0x01, _space_msg(a.shape)), (0x03, _dtype_msg(a.dtype))]
        if node.compact:
            raw = a.tobytes()
            msgs.append((0x08, struct.pack("<BBH", 3, 0, len(raw)) + raw))
        elif node.chunks is None:
            addr = self._alloc(a.tobytes())
            msgs.append((0x08, struct.pack("<BBQQ", 3, 1, addr, a.nbytes)))
        else:
            msgs.extend(self._chunked(a, node.chunks, node.filters))
        return self._header(msgs + self._attr_msgs(node.attrs))

    def _chunked(self, a, chunks, filters):
        rank, es = a.ndim, a.dtype.itemsize
        grid = [range(0, a.shape[k], chunks[k]) for k in range(rank)]
        entries = []
        for off in np.ndindex(*[len(g) for g in grid]):
            o = [off[k] * chunks[k] for k in range(rank)]
            blk = np.zeros(chunks, a.dtype)
            sl = tuple(slice(o[k], min(o[k] + chunks[k], a.shape[k])) for k in range(rank))
            part = a[sl]
            blk[tuple(slice(0, s) for s in part.shape)] = part
            raw = blk.tobytes()
            if "shuffle" in filters:
                raw = np.frombuffer(raw, np.uint8).reshape(-1, es).T.tobytes()
            if "deflate" in filters:
                raw = zlib.compress(raw, 6)
            entries.append((o, self._alloc(raw), len(raw)))
        tree = b"TREE" + struct.pack("<BBHQQ", 1, 0, len(entries), UNDEF, UNDEF)
        for o, addr, n in entries:
            tree += struct.pack("<II", n, 0) + b"".join(struct.pack("<Q", x) for x in o + [0])
            tree += struct.pack("<Q", addr)
        tree += struct.pack("<II", 0, 0) + b"".join(struct.pack("<Q", x) for x in list(a.shape) + [0])
        bt = self._alloc(tree)
        msgs = [(0x08, struct.pack("<BBBQ", 3, 2, rank + 1, bt)
                 + b"".join(struct.pack("<I", c) for c in list(chunks) + [es]))]
        if filters:
            fl = b""
            ids = [(2, [es]) if f == "shuffle" else (1, [6]) for f in filters]
            for fid, cd in ids:
                fl += struct.pack("<HHHH", fid, 0, 0, len(cd)) + b"".join(struct.pack("<I", c) for c in cd)
                if len(cd) % 2:
                    fl += b"\0" * 4
            msgs.append((0x0B, struct.pack("<BB6x", 1, len(ids)) + fl))
        return msgs

    # -- groups -----------------------------------------------------------
    def _group(self, node):
        kids = {name: self._object(child) for name, child in node.children.items()}
        if self.sb >= 2:
            heap = UNDEF if not self.dense_links else self._alloc(b"FRHP" + b"\0" * 60)
            msgs = [(0x02, struct.pack("<BBQQ", 0, 0, heap, UNDEF)), (0x0A, struct.pack("<BB", 0, 0))]
            for name, addr in sorted(kids.items()):
                nm = name.encode()
                msgs.append((0x06, struct.pack("<BBB", 1, 0, len(nm)) + nm + struct.pack("<Q", addr)))
            return self._header(msgs + self._attr_msgs(node.attrs))
        names = sorted(kids, key=lambda s: s.encode())
        heap_data = bytearray(b"\0" * 8)
        offs = {}
        for n in names:
            offs[n] = len(heap_data)
            heap_data += _pad8(n.encode() + b"\0")
        data_addr = self._alloc(bytes(heap_data))
        heap = self._alloc(b"HEAP" + struct.pack("<B3xQQQ", 0, len(heap_data), UNDEF, data_addr))
        # leaves: symbol-table nodes of snod_cap entries
        level = []
        for i in range(0, max(len(names), 1), self.snod_cap):
            part = names[i:i + self.snod_cap]
            body = b"".join(struct.pack("<QQII16x", offs[n], kids[n], 0, 0) for n in part)
            level.append((self._alloc(b"SNOD" + struct.pack("<BBH", 1, 0, len(part)) + body),
                          offs[part[-1]] if part else 0))
        depth = 0
        while True:
            nodes = []
            for i in range(0, len(level), self.bt_cap):
                part = level[i:i + self.bt_cap]
                tree = b"TREE" + struct.pack("<BBHQQ", 0, depth, len(part), UNDEF, UNDEF) + struct.pack("<Q", 0)
                for addr, last in part:
                    tree += struct.pack("<QQ", addr, last)
                nodes.append((self._alloc(tree), part[-1][1]))
            level, depth = nodes, depth + 1
            if len(level) == 1:
                break
        msgs = [(0x11, struct.pack("<QQ", level[0][0], heap))]
        return self._header(msgs + self._attr_msgs(node.attrs))

    def _object(self, node):
        return self._group(node) if node.data is None else self._dataset(node)

    def write(self, path, root):
        sb_size = 96 if self.sb < 2 else 48
        self.buf = bytearray(b"\0" * sb_size)
        root_addr = self._object(root)
        eof = len(self.buf)
        if self.sb < 2:
            sb = SIG + struct.pack("<BBBBBBBBHHI", 0, 0, 0, 0, 0, 8, 8, 0, 4, 16, 0)
            sb += struct.pack("<QQQQ", 0, UNDEF, eof, UNDEF)
            sb += struct.pack("<QQII16x", 0, root_addr, 0, 0)
        else:
            sb = SIG + struct.pack("<BBBB", 2, 8, 8, 0) + struct.pack("<QQQQ", 0, UNDEF, eof, root_addr) + b"\0" * 4
        self.buf[:len(sb)] = sb
        with open(path, "wb") as fh:
            fh.write(b"\0" * self.userblock + bytes(self.buf))


def write_eman2(path, images, attrs=None, **kw):
    """EMAN2 layout: /MDF/images/<n>/image plus EMAN.* attributes on the
    image group (int32 nx, ny, nz, as EMAN2 writes them)."""
    root = Node()
    for n, img in enumerate(images):
        img = np.asarray(img)
        g = root.group("/MDF/images/%d" % n)
        nz, ny, nx = (1,) * (3 - img.ndim) + img.shape
        g.attrs.update({"EMAN.nx": np.int32(nx), "EMAN.ny": np.int32(ny), "EMAN.nz": np.int32(nz),
                        "EMAN.apix_x": np.float32(1.0)})
        if attrs and n in attrs:
            g.attrs.update(attrs[n])
        opts = kw.get("dataset_options", {}).get(n, {})
        root.dataset("/MDF/images/%d/image" % n, img, **opts)
    Writer(**{k: v for k, v in kw.items() if k != "dataset_options"}).write(path, root)


def write_eman1(path, images, spacing=(1.0, 1.0, 1.0)):
    """Old EMAN layout: root attribute num_dataset, root datasets "0", "1", ...
    with spacing_row / spacing_col / spacing_sec attributes."""
    root = Node()
    root.attrs["num_dataset"] = np.int32(len(images))
    for n, img in enumerate(images):
        d = root.dataset("/%d" % n, np.asarray(img))
        d.attrs.update({"spacing_row": np.float32(spacing[0]), "spacing_col": np.float32(spacing[1]),
                        "spacing_sec": np.float32(spacing[2])})
    Writer().write(path, root)


def copy_case_as_hdf(d):
    """Beside a case written by gisspa_b200.synth.write_dataset in ``d``: its
    template stack as an EMAN2 file (templates.hdf), each micrograph as an
    old-style EMAN file holding it at image ``nn`` (dims (nx, ny) over the
    x-fastest pixels), a list naming them (micrographs_hdf.lst) and a config
    using both (config_hdf)."""
    import os

    from gisspa_b200 import formats
    cfg = formats.read_config(os.path.join(d, "config"))
    stack = formats.read_mrc(os.path.join(d, cfg.temp2d), -1)
    write_eman2(os.path.join(d, "templates.hdf"), [t for t in stack])
    lst = open(os.path.join(d, cfg.inlst)).read()
    for ln in lst.splitlines()[1:]:
        if not ln.strip():
            continue
        nn, name = ln.split("\t")[:2]
        img = formats.read_mrc(os.path.join(d, name), int(nn))
        ny, nx = img.shape
        flat = np.ascontiguousarray(img).reshape(nx, ny)  # EMAN1: dims (nx, ny) over x-fastest data
        write_eman1(os.path.join(d, name.replace(".mrc", ".hdf")), [flat] * (int(nn) + 1))
    with open(os.path.join(d, "micrographs_hdf.lst"), "w") as fh:
        fh.write(lst.replace(".mrc", ".hdf"))
    text = open(os.path.join(d, "config")).read()
    text = text.replace(cfg.temp2d, "templates.hdf").replace(cfg.inlst, "micrographs_hdf.lst")
    with open(os.path.join(d, "config_hdf"), "w") as fh:
        fh.write(text)
