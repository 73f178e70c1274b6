"""TEST INFRASTRUCTURE -- the CSV-to-NDJSON mapping, restated in Python.

The reference reads NDJSON only (its --csv flag is an output format,
crates/warpjq-core/src/output.rs:45-85), so there is no reference CSV reader
to pin against: this restatement defines the mapping the device converter
(warpjq_csv_convert) must reproduce byte for byte, and the NDJSON it yields
is then checked with the NDJSON oracle.  Parity of CSV input is therefore
relative to this mapping ("parity unpinned" against the reference).

Rules:
  - a '\\n' ends a row when an even number of '"' bytes precede it in the
    input; a '\\r' just before it is dropped; the input's end closes a last
    row that has no newline;
  - the first row is the header (a UTF-8 byte-order mark before it is
    dropped); every later row is one output line, an empty row an empty line;
  - fields are split at ','; a field starting with '"' is quoted: it runs to
    the next '"' that is not doubled, '""' inside it stands for '"', and the
    bytes after the closing quote up to the next ',' are kept as they are;
  - a row is an object with the header's names as keys, in order, over its
    first min(fields, names) fields;
  - an unquoted field that is a JSON number stays a number, an unquoted empty
    field is null, anything else is a JSON string.

Only tests and bench.py's CPU-baseline leg use it.
"""

from __future__ import annotations

import re

_NUMBER = re.compile(rb"-?(?:0|[1-9][0-9]*)(?:\.[0-9]+)?(?:[eE][+-]?[0-9]+)?\Z")
_SHORT = {0x22: b'\\"', 0x5C: b"\\\\", 0x0A: b"\\n", 0x0D: b"\\r", 0x09: b"\\t", 0x08: b"\\b", 0x0C: b"\\f"}


def json_string(raw: bytes) -> bytes:
    out = bytearray(b'"')
    for c in raw:
        if c in _SHORT:
            out += _SHORT[c]
        elif c < 0x20:
            out += b"\\u00%02x" % c
        else:
            out.append(c)
    out += b'"'
    return bytes(out)


def split_rows(data: bytes) -> list:
    """Rows as byte strings (without their newline)."""
    rows, start, inside = [], 0, False
    for i, c in enumerate(data):
        if c == 0x22:
            inside = not inside
        elif c == 0x0A and not inside:
            rows.append(data[start:i])
            start = i + 1
    if start < len(data):
        rows.append(data[start:])
    return rows


def split_fields(row: bytes) -> list:
    """(text, quoted) per field; text already unquoted."""
    if row.endswith(b"\r"):
        row = row[:-1]
    fields, p, n = [], 0, len(row)
    while True:
        if p < n and row[p] == 0x22:
            text = bytearray()
            p += 1
            while p < n:
                if row[p] == 0x22:
                    if p + 1 < n and row[p + 1] == 0x22:
                        text.append(0x22)
                        p += 2
                        continue
                    p += 1
                    break
                text.append(row[p])
                p += 1
            q = row.find(b",", p)
            q = n if q < 0 else q
            text += row[p:q]
            fields.append((bytes(text), True))
            p = q
        else:
            q = row.find(b",", p)
            q = n if q < 0 else q
            fields.append((row[p:q], False))
            p = q
        if p >= n:
            return fields
        p += 1


def value(text: bytes, quoted: bool) -> bytes:
    if not quoted and text == b"":
        return b"null"
    if not quoted and _NUMBER.match(text):
        return text
    return json_string(text)


def csv_to_ndjson(data: bytes) -> bytes:
    """The whole input's NDJSON (empty when there is no header row)."""
    if data.startswith(b"\xef\xbb\xbf"):
        data = data[3:]
    rows = split_rows(data)
    if not rows:
        return b""
    head = rows[0][:-1] if rows[0].endswith(b"\r") else rows[0]
    names = [t for t, _ in split_fields(head)] if head else []
    out = []
    for row in rows[1:]:
        if row in (b"", b"\r"):
            out.append(b"\n")
            continue
        parts = [json_string(names[k]) + b":" + value(t, q) for k, (t, q) in enumerate(split_fields(row))
                 if k < len(names)]
        out.append(b"{" + b",".join(parts) + b"}\n")
    return b"".join(out)
