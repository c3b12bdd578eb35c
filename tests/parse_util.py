"""CPU restatement of the reference's FASTA query parse (Sequences::GetNumberOfHeaders and
TReadFastaSequencesFromMem, Sequences.cpp:283-320, 57-214, as one pass over the file):
  - the file must start with '>' (the reference stops with "0 Headers found" otherwise);
  - each line starting with '>' is a header and starts a sequence (header kept with its '>',
    without a trailing '\\r');
  - other lines are appended to the current sequence without a trailing '\\r'; empty lines add
    nothing; an unterminated last line counts like the others;
  - sequences are uppercased (bytes above 96, as signed char, lose 32; Sequences.cpp:43-55)."""


def parse_fasta(text: bytes, uppercase: bool = True):
    if not text:
        return [], []
    if text[:1] != b">":
        raise ValueError("no FASTA header at the start of the file")
    seqs, hdrs = [], []
    for line in text.split(b"\n"):
        if line.endswith(b"\r"):
            line = line[:-1]
        if line.startswith(b">"):
            hdrs.append(line)
            seqs.append(bytearray())
        elif line.startswith(b"@"):
            raise ValueError("a line starts with '@'")
        else:
            seqs[-1] += line
    if uppercase:
        seqs = [bytes(c - 32 if 96 < c < 128 else c for c in s) for s in seqs]
    return [bytes(s) for s in seqs], hdrs
