"""SciDAC / ILDG gauge configurations in LIME files, read into (and written
from) the reference's BMXYIJ link layout on the device.

The reader covers what ``jaxqft/io/lime.py`` provides for the hot path
(record scan 69-103, SciDAC field metadata 163-224, decode 247-331, gauge
236-245 / 334-353, momentum 355-381, pseudofermion 384-422): LIME records
(USQCD LIME: 144-byte big-endian header = magic 0x456789ab, version, flags,
payload length, 128-byte type string; payloads padded to 8 bytes), the
SciDAC private file/record XML (dims; datatype, precision F/D, colours,
spins, typesize, datacount) or the ILDG format record (lx..lt), and the binary
payload: sites in SciDAC lexicographic order (x fastest), per site
``datacount`` items of big-endian (re, im) pairs.  The payload is decoded with
numpy, uploaded once, and permuted on the GPU into the t-fastest BMXYIJ layout
``[batch][mu][Lx][Ly][Lz][Lt][3][3]`` complex128 that the library consumes.

The writer produces the same record sequence (file XML, record XML,
binary data) so HMC configurations can be checkpointed and read back by
QIO-style readers.
"""

from __future__ import annotations

import re
import struct
from dataclasses import dataclass
from typing import Iterator, List, Optional, Sequence, Tuple

import numpy as np
import torch

MAGIC = 0x456789AB
HEADER = struct.Struct(">IHHQ128s")  # 144 bytes
MB_FLAG, ME_FLAG = 0x8000, 0x4000


@dataclass(frozen=True)
class Record:
    index: int
    offset: int      # header offset
    flags: int
    nbytes: int
    type: str

    @property
    def payload(self) -> int:
        return self.offset + HEADER.size


@dataclass(frozen=True)
class Field:
    datatype: str
    precision: str
    colors: int
    spins: int
    typesize: int
    datacount: int
    dims: Tuple[int, ...]
    recordtype: Optional[int]
    binary: Record


def records(path) -> Iterator[Record]:
    """Scan the LIME records of a file."""
    with open(path, "rb") as f:
        off, idx = 0, 0
        while True:
            hdr = f.read(HEADER.size)
            if not hdr:
                return
            if len(hdr) != HEADER.size:
                raise ValueError(f"{path}: truncated LIME header at byte {off}")
            magic, _ver, flags, nbytes, tname = HEADER.unpack(hdr)
            if magic != MAGIC:
                raise ValueError(f"{path}: not a LIME record at byte {off} (magic {magic:#x})")
            yield Record(idx, off, flags, nbytes, tname.split(b"\0", 1)[0].decode("ascii", "replace"))
            off += HEADER.size + nbytes + ((-nbytes) & 7)
            f.seek(off)
            idx += 1


def _read(path, rec: Record) -> bytes:
    with open(path, "rb") as f:
        f.seek(rec.payload)
        data = f.read(rec.nbytes)
    if len(data) != rec.nbytes:
        raise ValueError(f"{path}: record {rec.index} ({rec.type}) is truncated")
    return data


def _tag(xml: str, name: str) -> Optional[str]:
    m = re.search(rf"<{name}(?:\s[^>]*)?>(.*?)</{name}>", xml, re.S)
    return None if m is None else m.group(1).strip()


def _int(text: Optional[str], default):
    try:
        return int(text) if text is not None else default
    except ValueError:
        return default


def fields(path) -> List[Field]:
    """SciDAC fields of a file: each private record XML with its binary payload."""
    recs = list(records(path))
    xml = {r.index: _read(path, r).decode("utf-8", "replace") for r in recs
           if "xml" in r.type or r.type == "ildg-format"}
    dims: Tuple[int, ...] = ()
    for r in recs:
        if r.type == "scidac-private-file-xml":
            d = _tag(xml[r.index], "dims")
            if d:
                dims = tuple(int(v) for v in d.split())
    if not dims:
        for r in recs:
            if r.type == "ildg-format":
                vals = [_tag(xml[r.index], t) for t in ("lx", "ly", "lz", "lt")]
                if all(v is not None for v in vals):
                    dims = tuple(int(v) for v in vals)
    out = []
    for i, r in enumerate(recs):
        if r.type != "scidac-private-record-xml":
            continue
        x = xml[r.index]
        binary = next((b for b in recs[i + 1:] if b.type in ("ildg-binary-data", "scidac-binary-data")), None)
        if binary is None:
            continue
        out.append(Field(datatype=_tag(x, "datatype") or "", precision=(_tag(x, "precision") or "F").upper(),
                         colors=_int(_tag(x, "colors"), 0), spins=_int(_tag(x, "spins"), 0),
                         typesize=_int(_tag(x, "typesize"), 0), datacount=_int(_tag(x, "datacount"), 1),
                         dims=dims, recordtype=_int(_tag(x, "recordtype"), None), binary=binary))
    return out


def _site_items(path, fd: Field) -> Tuple[np.ndarray, int]:
    """Payload as complex128 [V][datacount][n] (SciDAC site order), n = complex per item."""
    if fd.precision not in ("F", "D"):
        raise ValueError(f"unsupported SciDAC precision {fd.precision!r}")
    word = 4 if fd.precision == "F" else 8
    if fd.typesize % (2 * word):
        raise ValueError(f"typesize {fd.typesize} is not a whole number of complex {fd.precision} values")
    ncplx = fd.typesize // (2 * word)
    raw = np.frombuffer(_read(path, fd.binary), dtype=">f4" if word == 4 else ">f8")
    if not fd.dims:
        raise ValueError("the file carries no lattice dimensions")
    vol = int(np.prod(fd.dims))
    if raw.size != vol * fd.datacount * ncplx * 2:
        raise ValueError(f"binary payload of {raw.size} words does not match V={vol} x {fd.datacount} x "
                         f"{ncplx} complex values")
    re_im = raw.astype(np.float64).reshape(vol, fd.datacount, ncplx, 2)
    return re_im[..., 0] + 1j * re_im[..., 1], ncplx


def _to_device_layout(items: np.ndarray, dims: Sequence[int], inner: Tuple[int, ...], device) -> torch.Tensor:
    """[V (x fastest)][datacount][...] -> device [datacount][Lx][Ly][Lz][Lt][...]."""
    nd = len(dims)
    t = torch.from_numpy(np.ascontiguousarray(items)).to(device)
    t = t.reshape(*reversed(tuple(dims)), items.shape[1], *inner)   # [Lt][Lz][Ly][Lx][dc][...]
    perm = (nd,) + tuple(range(nd - 1, -1, -1)) + tuple(range(nd + 1, t.dim()))
    return t.permute(*perm).contiguous()


def load_gauge(path, field_index: int = 0, batch_size: int = 1, device=None) -> torch.Tensor:
    """Gauge links [batch][mu][Lx][Ly][Lz][Lt][Nc][Nc] complex128 on the device
    (lime.py:334-353 decode_scidac_gauge)."""
    device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    fd = fields(path)[field_index]
    if "ColorMatrix" not in fd.datatype:
        raise ValueError(f"expected a ColorMatrix field, found {fd.datatype!r}")
    items, ncplx = _site_items(path, fd)
    nc = fd.colors
    if ncplx != nc * nc:
        raise ValueError(f"ColorMatrix item of {ncplx} complex values, expected {nc * nc}")
    U = _to_device_layout(items, fd.dims, (nc, nc), device)
    return U[None].repeat(int(batch_size), *([1] * U.dim())) if batch_size != 1 else U[None]


def load_momentum(path, field_index: int = 0, batch_size: int = 1, device=None):
    """Momenta stored like gauge links (lime.py:355-381), with the traceless
    anti-Hermitian diagnostics of the reference."""
    P = load_gauge(path, field_index, batch_size, device)
    Pd = P.conj().transpose(-1, -2)
    nrm = float(torch.linalg.vector_norm(P))
    tr = torch.diagonal(P, dim1=-2, dim2=-1).sum(-1).abs()
    info = {"rel_antihermitian_error": float(torch.linalg.vector_norm(P + Pd)) / nrm if nrm > 0 else 0.0,
            "mean_abs_trace": float(tr.mean()), "max_abs_trace": float(tr.max())}
    return P, info


def load_fermion(path, field_index: Optional[int] = None, batch_size: int = 1, device=None):
    """Dirac fermion [batch][Lx][Ly][Lz][Lt][Ns][Nc] (lime.py:384-422); without an
    index, the first field with spins and colours and record type 0."""
    device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    fl = fields(path)
    if field_index is None:
        cand = [i for i, f in enumerate(fl) if f.spins > 0 and f.colors > 0 and f.recordtype in (0, None)]
        if not cand:
            raise ValueError("no pseudofermion-like field in the file; pass field_index")
        field_index = cand[0]
    fd = fl[field_index]
    items, ncplx = _site_items(path, fd)
    if ncplx != fd.spins * fd.colors:
        raise ValueError(f"fermion item of {ncplx} complex values, expected {fd.spins * fd.colors}")
    F = _to_device_layout(items, fd.dims, (fd.spins, fd.colors), device)  # [dc][*L][s][c]
    F = F[0] if fd.datacount == 1 else F.movedim(0, -3)
    F = F[None]
    return (F.repeat(int(batch_size), *([1] * (F.dim() - 1))) if batch_size != 1 else F), fd


# ----------------------------------------------------------------------------- writer
def _record(f, type_name: str, payload: bytes, flags: int) -> None:
    f.write(HEADER.pack(MAGIC, 1, flags, len(payload), type_name.encode("ascii")))
    f.write(payload)
    f.write(b"\0" * ((-len(payload)) & 7))


def _write_field(path, sites: np.ndarray, dims, datatype: str, precision: str, colors: int, spins: int,
                 datacount: int) -> None:
    word = {"F": 4, "D": 8}[precision]
    reim = np.stack([sites.real, sites.imag], axis=-1).astype(">f4" if word == 4 else ">f8")
    typesize = int(np.prod(sites.shape[len(dims) + 1:])) * 2 * word  # bytes of one item (re, im pairs)
    dims_txt = " ".join(str(int(d)) for d in dims)
    file_xml = (f'<?xml version="1.0"?><scidacFile><version>1.1</version><spacetime>{len(dims)}</spacetime>'
                f"<dims>{dims_txt} </dims><volfmt>0</volfmt></scidacFile>")
    rec_xml = (f'<?xml version="1.0"?><scidacRecord><version>1.1</version><date>unknown</date>'
               f"<recordtype>0</recordtype><datatype>{datatype}</datatype>"
               f"<precision>{precision}</precision><colors>{colors}</colors><spins>{spins}</spins>"
               f"<typesize>{typesize}</typesize><datacount>{datacount}</datacount></scidacRecord>")
    with open(path, "wb") as f:
        _record(f, "scidac-private-file-xml", file_xml.encode(), MB_FLAG | ME_FLAG)
        _record(f, "scidac-private-record-xml", rec_xml.encode(), MB_FLAG)
        _record(f, "scidac-binary-data", reim.tobytes(), ME_FLAG)


def save_fermion(path, psi, precision: str = "D") -> None:
    """Write one Dirac fermion [Lx][Ly][Lz][Lt][Ns][Nc] (or [1][...]) as SciDAC LIME."""
    if isinstance(psi, torch.Tensor):
        psi = psi.detach().cpu().numpy()
    psi = np.asarray(psi)
    if psi.ndim == 7:
        psi = psi[0]
    nd = psi.ndim - 2
    ns, nc = psi.shape[-2:]
    sites = np.transpose(psi, tuple(range(nd - 1, -1, -1)) + (nd, nd + 1))[..., None, :, :]
    p = precision.upper()
    _write_field(path, sites, psi.shape[:nd], f"QDP_{p}{nc}_DiracFermion", p, nc, ns, 1)


def save_gauge(path, U, precision: str = "D") -> None:
    """Write one configuration U [mu][Lx][Ly][Lz][Lt][3][3] (or [1][mu]...) as a
    SciDAC LIME file: file XML (dims), record XML (QDP ColorMatrix, datacount 4),
    binary data in SciDAC site order, big-endian."""
    if isinstance(U, torch.Tensor):
        U = U.detach().cpu().numpy()
    U = np.asarray(U)
    if U.ndim == 8:
        if U.shape[0] != 1:
            raise ValueError("save_gauge writes one configuration")
        U = U[0]
    nd = U.ndim - 3
    dims = U.shape[1:1 + nd]
    nc = U.shape[-1]
    precision = precision.upper()
    # [mu][Lx..Lt][a][b] -> [Lt][Lz][Ly][Lx][mu][a][b] (x fastest)
    sites = np.transpose(U, tuple(range(nd, 0, -1)) + (0, nd + 1, nd + 2))
    _write_field(path, sites, dims, f"QDP_{precision}{nc}_ColorMatrix", precision, nc, 0, U.shape[0])
