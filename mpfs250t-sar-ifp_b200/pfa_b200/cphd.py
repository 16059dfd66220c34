"""CPHD 1.0 phase-history files without sarpy: the reader the reference reaches through
``sarpy.io.phase_history.converter.open_phase_history`` (src/form_image_pfa.py:37, 305-347;
mpfs/host/sar_pipeline.py:118-135), and a writer for synthetic scenes.

Only what the focusing path reads is interpreted: the file header's block offsets, the XML's
Global/DomainType and SGN, SceneCoordinates/ReferenceSurface/Planar uIAX and uIAY, the Data section
(signal format, channels, vectors, samples, byte offsets, NumBytesPVP) and the PVP layout (field
offsets in 8-byte words, big-endian F8 values); signal arrays in CF8 (big-endian complex float32), CI4 or
CI2 (big-endian signed integer I/Q pairs).

``CphdReader`` offers the reader methods the reference calls (``get_data_size_as_tuple``,
``read_pvp_variable``, ``read_chip``, ``cphd_meta.Global.SGN``,
``cphd_meta.SceneCoordinates.ReferenceSurface.Planar.uIAX/uIAY``, ``close``), so
``geometry.prepare_tables_fast(reader, reader.cphd_meta)`` and the reference's own ``prepare_tables`` run
on it unchanged, plus ``read_signal_into`` to fill a caller's (pinned) complex64 buffer in one pass
(the big-endian samples are converted while they are copied).  ``write_cphd`` writes the same subset,
which is what the tests and the synthetic benchmark scenes use: no CPHD collect is available here.
"""
from __future__ import annotations

import re
import xml.etree.ElementTree as ET
from pathlib import Path
from types import SimpleNamespace

import numpy as np

_SIG_DTYPES = {"CF8": np.dtype(">c8"), "CI4": np.dtype([("i", ">i2"), ("q", ">i2")]),
               "CI2": np.dtype([("i", "i1"), ("q", "i1")])}


def _local(tag):
    return tag.rsplit("}", 1)[-1]


def _find(node, path):
    """Namespace-agnostic child lookup along a '/'-separated path (None if missing)."""
    for name in path.split("/"):
        if node is None:
            return None
        node = next((c for c in node if _local(c.tag) == name), None)
    return node


def _xyz(node):
    return SimpleNamespace(X=float(_find(node, "X").text), Y=float(_find(node, "Y").text),
                           Z=float(_find(node, "Z").text))


class CphdReader:
    """Reader of one CPHD 1.0 file (see the module docstring for the subset)."""

    def __init__(self, path):
        self.path = Path(path)
        self._fh = open(self.path, "rb")
        head = b""
        while not head.endswith(b"\f\n"):
            ch = self._fh.read(1)
            if not ch:
                raise ValueError(f"{path}: no CPHD file header terminator")
            head += ch
        lines = head.decode("ascii").splitlines()
        if not lines or not lines[0].startswith("CPHD/"):
            raise ValueError(f"{path}: not a CPHD file")
        self.version = lines[0][5:]
        self.header = {}
        for ln in lines[1:]:
            m = re.match(r"\s*([A-Z_]+)\s*:=\s*(.*?)\s*$", ln)
            if m:
                self.header[m.group(1)] = m.group(2)
        self._fh.seek(int(self.header["XML_BLOCK_BYTE_OFFSET"]))
        self.xml = self._fh.read(int(self.header["XML_BLOCK_SIZE"])).decode("utf-8")
        root = ET.fromstring(self.xml)
        glob = _find(root, "Global")
        planar = _find(root, "SceneCoordinates/ReferenceSurface/Planar")
        self.cphd_meta = SimpleNamespace(
            Global=SimpleNamespace(DomainType=_find(glob, "DomainType").text.strip(),
                                   SGN=int(_find(glob, "SGN").text)),
            SceneCoordinates=SimpleNamespace(ReferenceSurface=SimpleNamespace(Planar=SimpleNamespace(
                uIAX=_xyz(_find(planar, "uIAX")), uIAY=_xyz(_find(planar, "uIAY"))))))
        data = _find(root, "Data")
        self.signal_format = _find(data, "SignalArrayFormat").text.strip()
        if self.signal_format not in _SIG_DTYPES:
            raise ValueError(f"{path}: signal format {self.signal_format} not supported")
        self.num_bytes_pvp = int(_find(data, "NumBytesPVP").text)
        self.channels = []
        for ch in data:
            if _local(ch.tag) != "Channel":
                continue
            self.channels.append(dict(
                id=_find(ch, "Identifier").text.strip(), num_vectors=int(_find(ch, "NumVectors").text),
                num_samples=int(_find(ch, "NumSamples").text),
                signal_offset=int(_find(ch, "SignalArrayByteOffset").text),
                pvp_offset=int(_find(ch, "PVPArrayByteOffset").text)))
        self.pvp_fields = {}
        for fld in _find(root, "PVP"):
            name = _local(fld.tag)
            if name == "AddedPVP":
                name = _find(fld, "Name").text.strip()
            self.pvp_fields[name] = (int(_find(fld, "Offset").text), int(_find(fld, "Size").text),
                                     _find(fld, "Format").text.strip())
        self._pvp = {}

    # ---------------------------------------------------------------- the sarpy reader subset
    def get_data_size_as_tuple(self):
        return tuple((c["num_vectors"], c["num_samples"]) for c in self.channels)

    def _pvp_block(self, index):
        if index not in self._pvp:
            c = self.channels[index]
            words = self.num_bytes_pvp // 8
            off = int(self.header["PVP_BLOCK_BYTE_OFFSET"]) + c["pvp_offset"]
            self._pvp[index] = np.fromfile(self.path, dtype=">f8", count=c["num_vectors"] * words,
                                           offset=off).reshape(c["num_vectors"], words)
        return self._pvp[index]

    def read_pvp_variable(self, name, index=0):
        off, size, fmt = self.pvp_fields[name]
        if not all(f.endswith("F8") for f in fmt.split(";") if f):
            raise ValueError(f"PVP {name}: format {fmt} not supported")
        block = self._pvp_block(index)
        v = block[:, off:off + size].astype(np.float64)
        return v[:, 0].copy() if size == 1 else v.copy()

    def _signal_map(self, index):
        c = self.channels[index]
        off = int(self.header["SIGNAL_BLOCK_BYTE_OFFSET"]) + c["signal_offset"]
        return np.memmap(self.path, dtype=_SIG_DTYPES[self.signal_format], mode="r", offset=off,
                         shape=(c["num_vectors"], c["num_samples"]))

    @staticmethod
    def _to_c64(a):
        if a.dtype.names:
            return (a["i"].astype(np.float32) + 1j * a["q"].astype(np.float32)).astype(np.complex64)
        return a.astype(np.complex64)

    def read_chip(self, rows, cols, index=0):
        """Signal of channel ``index`` at rows (start, stop, step) and cols (start, stop, step)."""
        mm = self._signal_map(index)
        out = self._to_c64(mm[slice(*rows), slice(*cols)])
        del mm
        return out

    def read_signal_into(self, out, index=0, rows=None, cols=None):
        """Copy the (decimated) signal into ``out`` (complex64, C-contiguous, e.g. pinned host memory),
        converting from the file's big-endian format in the same pass.  Returns ``out``."""
        c = self.channels[index]
        rows = rows or (0, c["num_vectors"], 1)
        cols = cols or (0, c["num_samples"], 1)
        mm = self._signal_map(index)
        src = mm[slice(*rows), slice(*cols)]
        if out.shape != src.shape or out.dtype != np.complex64:
            raise ValueError(f"out must be complex64 {src.shape}")
        if src.dtype.names:
            out.real[...] = src["i"]
            out.imag[...] = src["q"]
        else:
            np.copyto(out, src, casting="same_kind")
        del mm
        return out

    def close(self):
        if self._fh:
            self._fh.close()
            self._fh = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def open_phase_history(path):
    """Drop-in for sarpy.io.phase_history.converter.open_phase_history on CPHD 1.0 files."""
    return CphdReader(path)


# ----------------------------------------------------------------------------- writer
_PVP_LAYOUT = [("TxTime", 1), ("TxPos", 3), ("TxVel", 3), ("RcvTime", 1), ("RcvPos", 3), ("RcvVel", 3),
               ("SRPPos", 3), ("SC0", 1), ("SCSS", 1), ("FX1", 1), ("FX2", 1)]


def write_cphd(path, signal, tx, rcv, srp, sc0, scss, uiax, uiay, sgn=-1, iarp=None, fmt="CF8"):
    """Write a single-channel FX-domain CPHD 1.0 file of the focusing subset.  signal: (m, n) complex;
    tx, rcv, srp: (m, 3) ECEF; sc0, scss: (m,) Hz.  fmt: "CF8" (complex float32) or "CI4" (int16 I/Q,
    the signal rounded)."""
    signal = np.asarray(signal)
    m, n = signal.shape
    words = sum(s for _, s in _PVP_LAYOUT)
    pvp = np.zeros((m, words), ">f8")
    cols = {"TxPos": tx, "RcvPos": rcv, "SRPPos": srp, "SC0": sc0, "SCSS": scss,
            "FX1": sc0, "FX2": np.asarray(sc0) + (n - 1) * np.asarray(scss)}
    off = 0
    pvp_xml = []
    for name, size in _PVP_LAYOUT:
        if name in cols:
            pvp[:, off:off + size] = np.asarray(cols[name], np.float64).reshape(m, size)
        f = "X=F8;Y=F8;Z=F8;" if size == 3 else "F8"
        pvp_xml.append(f"<{name}><Offset>{off}</Offset><Size>{size}</Size><Format>{f}</Format></{name}>")
        off += size
    if fmt == "CF8":
        sig = np.ascontiguousarray(signal, ">c8")
    elif fmt == "CI4":
        sig = np.empty((m, n), _SIG_DTYPES["CI4"])
        sig["i"] = np.clip(np.rint(signal.real), -32768, 32767)
        sig["q"] = np.clip(np.rint(signal.imag), -32768, 32767)
    else:
        raise ValueError("fmt must be CF8 or CI4")
    ip = np.asarray(iarp if iarp is not None else srp[0], np.float64)
    v = lambda t, a: f"<{t}><X>{float(a[0])!r}</X><Y>{float(a[1])!r}</Y><Z>{float(a[2])!r}</Z></{t}>"   # noqa: E731
    xml = ('<?xml version="1.0" encoding="UTF-8"?>\n'
           '<CPHD xmlns="http://api.nsgreg.nga.mil/schema/cphd/1.0.1">'
           "<CollectionID><CollectorName>synthetic</CollectorName></CollectionID>"
           f"<Global><DomainType>FX</DomainType><SGN>{int(sgn)}</SGN></Global>"
           f"<SceneCoordinates><EarthModel>WGS_84</EarthModel><IARP>{v('ECF', ip)}</IARP>"
           f"<ReferenceSurface><Planar>{v('uIAX', uiax)}{v('uIAY', uiay)}</Planar></ReferenceSurface>"
           "</SceneCoordinates>"
           f"<Data><SignalArrayFormat>{fmt}</SignalArrayFormat><NumBytesPVP>{8 * words}</NumBytesPVP>"
           f"<NumCPHDChannels>1</NumCPHDChannels><Channel><Identifier>1</Identifier>"
           f"<NumVectors>{m}</NumVectors><NumSamples>{n}</NumSamples>"
           "<SignalArrayByteOffset>0</SignalArrayByteOffset><PVPArrayByteOffset>0</PVPArrayByteOffset>"
           "</Channel><NumSupportArrays>0</NumSupportArrays></Data>"
           f"<PVP>{''.join(pvp_xml)}</PVP></CPHD>").encode("utf-8")
    sizes = {"XML": len(xml), "PVP": pvp.nbytes, "SIGNAL": sig.nbytes}
    offs = {"XML": 0, "PVP": 0, "SIGNAL": 0}
    for _ in range(4):          # the header's length depends on the offsets it states
        head = (f"CPHD/1.0.1\nXML_BLOCK_SIZE := {sizes['XML']}\nXML_BLOCK_BYTE_OFFSET := {offs['XML']}\n"
                f"PVP_BLOCK_SIZE := {sizes['PVP']}\nPVP_BLOCK_BYTE_OFFSET := {offs['PVP']}\n"
                f"SIGNAL_BLOCK_SIZE := {sizes['SIGNAL']}\nSIGNAL_BLOCK_BYTE_OFFSET := {offs['SIGNAL']}\n"
                "CLASSIFICATION := UNCLASSIFIED\nRELEASE_INFO := UNRESTRICTED\n\f\n").encode("ascii")
        x0 = len(head)
        p0 = (x0 + len(xml) + 2 + 7) // 8 * 8                # XML, its "\f\n", 8-byte aligned PVP
        s0 = p0 + pvp.nbytes
        if (offs["XML"], offs["PVP"], offs["SIGNAL"]) == (x0, p0, s0):
            break
        offs = {"XML": x0, "PVP": p0, "SIGNAL": s0}
    with open(path, "wb") as fh:
        fh.write(head)
        fh.write(xml)
        fh.write(b"\f\n")
        fh.write(b"\0" * (offs["PVP"] - fh.tell()))
        fh.write(pvp.tobytes())
        fh.write(sig.tobytes())
    return path


def write_scene(path, scene, fmt="CF8"):
    """A synth.Scene (with its signal) as a CPHD file."""
    return write_cphd(path, scene.signal, scene.tx, scene.rcv, scene.srp, scene.sc0, scene.scss,
                      scene.uiax, scene.uiay, scene.sgn, fmt=fmt)
