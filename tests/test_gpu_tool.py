"""mirage_gpu, the drop-in program: the reference's configuration file and CLI overrides, a
FASTA reference or .mhm index in, the reference-format result logs out -- identical to the
reference's own results_Raw.log for the same inputs."""
import glob
import gzip
import os
import subprocess

import pytest

import mirage_b200 as M

pytestmark = pytest.mark.gpu

TOOL = os.path.join(os.path.dirname(M.LIB_PATH), "mirage_gpu")

CFG = """# MirAge configuration (the keys the classification path reads)
Query:{query}
Reference:{reference}
considerthreshold:31
OutputPath:{out}
output_firstresults_only:1
Hashmap_Load_Reference_Memory_UsageMode:extreme
Hashmap_Load_Hashmap_Percentage:100
UltraFastMode:Sensitive
output_save_hashmap_database:1
LogThreshold_HighSensitivity:0.4
LogThreshold_HighPrecision:1
LogThreshold_Balanced:0.7
"""


def run_tool(tmp, cfg_text, *args):
    cfg = os.path.join(tmp, "mirage.cfg")
    open(cfg, "w").write(cfg_text)
    p = subprocess.run([TOOL, "-cfg", cfg, *args], capture_output=True, text=True)
    assert p.returncode == 0, p.stderr + p.stdout
    dirs = sorted(glob.glob(os.path.join(tmp, "out", "results_*")))
    return dirs[-1]


def test_tool_from_fasta_and_from_mhm(golden, tmp_path):
    g = golden("plain")
    tmp = str(tmp_path)
    os.makedirs(os.path.join(tmp, "out"))
    refs = os.path.join(tmp, "refs.fasta")
    reads = os.path.join(tmp, "reads.fasta")
    g.refs.write_fasta(refs)
    g.reads.write_fasta(reads)
    exp = gzip.open(os.path.join(g.dir, "raw.log.gz"), "rb").read()
    # FASTA reference: indexed on the fly, index saved next to the logs
    d = run_tool(tmp, CFG.format(query=reads, reference=refs, out=os.path.join(tmp, "out")))
    assert open(os.path.join(d, "results_Raw.log"), "rb").read() == exp
    saved = os.path.join(d, "hashmap_refs.mhm")
    assert os.path.exists(saved)
    assert open(saved, "rb").read() == g.image.tobytes()  # the reference builder's bytes
    # .mhm reference through a CLI override of the configuration's Reference
    import time
    time.sleep(1.1)  # results folders are named by the second
    d2 = run_tool(tmp, CFG.format(query="/nonexistent", reference=refs, out=os.path.join(tmp, "out")),
                  "-reference", saved, "-input", reads)
    assert open(os.path.join(d2, "results_Raw.log"), "rb").read() == exp
    # batches of 1,500 reads: each batch's logs are written by a thread while the next batch is
    # classified; the log is the same, in the same order
    time.sleep(1.1)
    d3 = run_tool(tmp, CFG.format(query=reads, reference=saved, out=os.path.join(tmp, "out")), "-GPU_BatchReads", "1500")
    assert open(os.path.join(d3, "results_Raw.log"), "rb").read() == exp
