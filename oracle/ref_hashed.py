"""Builds _ref/cudaplex_hashed: the reference CudaPlex with the project's plex hash added.

CHECKER ONLY (test infrastructure, untimed, never shipped).  The reference
never materialises an output set: it only increments a counter at its two
counting sites in the BNB kernel (src/device_funcs.cu:1585 for a leaf with an
empty candidate set, :1716 for P u C reported whole).  To pin the project hash
(kplex_common.h: per set x = splitmix64(seed ^ |S|), x = splitmix64(x ^ v) for
the sorted original ids v, summed mod 2^64) against the reference itself, this
script

  1. copies main.cu, inc/ and src/ of the reference (given by --ref, read only)
     into _ref/hashed_src/ (the reference tree itself is never written);
  2. adds, at exactly those two sites and nowhere else, a call that maps the
     set's local ids to peeled ids through the root's d_blk slot
     (d_blk + t.idx * MAX_BLK_SIZE, filled by decompose, src:49 and 255) and
     peeled ids to input ids through the host's peel maps, sorts them and adds
     the set's hash to a device accumulator;
  3. records the peel maps on the host after each peelGraph call
     (inc/host_funcs.h:749 and 823; peelGraph keeps the vertices with
     mark[i] == true in ascending order, host:60-68) and prints
     "Plex hash: 0x..." after the reference's own result lines (host:1156-1157);
  4. compiles the copy with the reference's own flags (compile.sh:5) for sm_100a.

Every edit is an exact-anchor substitution that must match once, so a changed
reference fails loudly instead of being patched in the wrong place.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))

DEVICE_PRELUDE = r'''
// ---- added by oracle/ref_hashed.py (checker copy; not part of the reference) ----
__device__ unsigned long long g_ref_hash = 0;
__device__ const unsigned int* g_ref_orig = nullptr;

__device__ __forceinline__ unsigned long long ref_mix64(unsigned long long z)
{
  z += 0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

// One thread: the set a[0..na) + b[0..nb) of local ids of the root whose d_blk
// slot is blk.  Peel maps keep the input order, so sorting peeled ids sorts
// the input ids.
__device__ __noinline__ void ref_hash_add(const unsigned int* blk, const unsigned int* a, unsigned int na,
                                          const unsigned int* b, unsigned int nb)
{
  unsigned int ids[1024];
  unsigned int m = 0;
  for (unsigned int i = 0; i < na && m < 1024; ++i) ids[m++] = blk[a[i]];
  for (unsigned int i = 0; i < nb && m < 1024; ++i) ids[m++] = blk[b[i]];
  for (unsigned int i = 1; i < m; ++i)
  {
    const unsigned int v = ids[i];
    unsigned int j = i;
    while (j > 0 && ids[j - 1] > v) { ids[j] = ids[j - 1]; --j; }
    ids[j] = v;
  }
  unsigned long long x = ref_mix64(0x6b706c6578b200ULL ^ (unsigned long long)m);
  for (unsigned int i = 0; i < m; ++i) x = ref_mix64(x ^ (unsigned long long)g_ref_orig[ids[i]]);
  atomicAdd(&g_ref_hash, x);
}

void ref_hash_set_orig(const unsigned int* h_orig, int n)
{
  unsigned int* d = nullptr;
  cudaMalloc(&d, (n > 0 ? n : 1) * sizeof(unsigned int));
  if (n > 0) cudaMemcpy(d, h_orig, n * sizeof(unsigned int), cudaMemcpyHostToDevice);
  const unsigned int* dc = d;
  cudaMemcpyToSymbol(g_ref_orig, &dc, sizeof(dc));
  unsigned long long z = 0;
  cudaMemcpyToSymbol(g_ref_hash, &z, sizeof(z));
}

unsigned long long ref_hash_get()
{
  unsigned long long h = 0;
  cudaMemcpyFromSymbol(&h, g_ref_hash, sizeof(h));
  return h;
}
// ---- end of addition ----
'''

HOST_DECL = r'''
// ---- added by oracle/ref_hashed.py (checker copy) ----
void ref_hash_set_orig(const unsigned int* h_orig, int n);
unsigned long long ref_hash_get();
// ----
'''


def sub_once(text: str, anchor: str, repl: str, where: str) -> str:
    n = text.count(anchor)
    if n != 1:
        raise SystemExit(f"{where}: anchor found {n} times, expected once: {anchor!r}")
    return text.replace(anchor, repl)


def patch_device(path: str) -> None:
    text = open(path).read()
    head = '#include "../inc/device_funcs.h"\n\n'
    text = sub_once(text, head, head + DEVICE_PRELUDE + "\n", "device_funcs.cu prelude")
    start = text.index("__global__ void BNB(int i,")
    end = text.index("__device__ int commonEle(", start)
    body = text[start:end]
    site1 = "if(lane_id == 0) atomicAdd(&plex_count[0], 1);"
    site2 = "if (lane_id == 0) atomicAdd(&plex_count[0], 1);"
    body = sub_once(body, site1,
                    "if(lane_id == 0) { atomicAdd(&plex_count[0], 1); "
                    "ref_hash_add(d_blk + t.idx * MAX_BLK_SIZE, plex, PlexSz, cand, 0); }",
                    "BNB count site (empty candidate set)")
    body = sub_once(body, site2,
                    "if (lane_id == 0) { atomicAdd(&plex_count[0], 1); "
                    "ref_hash_add(d_blk + t.idx * MAX_BLK_SIZE, plex, PlexSz, cand, CandSz); }",
                    "BNB count site (P u C)")
    text = text[:start] + body + text[end:]
    open(path, "w").write(text)


def patch_host(path: str) -> None:
    text = open(path).read()
    text = sub_once(text, '#include "free_memories.h"\n', '#include "free_memories.h"\n' + HOST_DECL, "host decl")
    first = "graph<intT> peelG = peelGraph(g, mark, resNei);"
    text = sub_once(text, first, first + "\n    std::vector<unsigned int> ref_orig;"
                    "\n    for (int i_ = 0; i_ < g.n; ++i_) if (mark[i_]) ref_orig.push_back((unsigned int)i_);",
                    "first peel")
    second = "peelG = peelGraph(peelG, mark, resNei);\npn = peelG.n;"
    text = sub_once(text, second,
                    "{ const int pn_before_ = peelG.n;\n"
                    "peelG = peelGraph(peelG, mark, resNei);\n"
                    "std::vector<unsigned int> o2_;\n"
                    "for (int i_ = 0; i_ < pn_before_; ++i_) if (mark[i_]) o2_.push_back(ref_orig[i_]);\n"
                    "ref_orig.swap(o2_); }\npn = peelG.n;", "truss re-peel")
    loop = "for (int i = 0; i < (pn/WARPS)+1; i++)"
    text = sub_once(text, loop, "ref_hash_set_orig(ref_orig.data(), (int)ref_orig.size());\n    " + loop, "search loop")
    last = 'printf("Total tasks generated: %u\\n", h_global);'
    text = sub_once(text, last, last + '\n    printf("Plex hash: 0x%016llx\\n", ref_hash_get());', "result lines")
    open(path, "w").write(text)


def main() -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--ref", required=True, help="root of the reference project (read only)")
    ap.add_argument("--out", default=os.path.join(HERE, "_ref"))
    ap.add_argument("--arch", default="sm_100a")
    a = ap.parse_args()
    src = os.path.join(a.out, "hashed_src")
    if os.path.isdir(src):
        shutil.rmtree(src)
    os.makedirs(src)
    shutil.copy(os.path.join(a.ref, "main.cu"), src)
    shutil.copytree(os.path.join(a.ref, "inc"), os.path.join(src, "inc"))
    shutil.copytree(os.path.join(a.ref, "src"), os.path.join(src, "src"))
    for root, _, files in os.walk(src):
        for f in files:
            os.chmod(os.path.join(root, f), 0o644)
    patch_device(os.path.join(src, "src", "device_funcs.cu"))
    patch_host(os.path.join(src, "inc", "host_funcs.h"))
    exe = os.path.join(a.out, "cudaplex_hashed")
    cmd = ["nvcc", f"-arch={a.arch}", "--maxrregcount=64", "--extended-lambda", "-Xcompiler", "-fopenmp",
           os.path.join(src, "src", "device_funcs.cu"), os.path.join(src, "main.cu"), "-o", exe]
    print(" ".join(cmd), flush=True)
    return subprocess.call(cmd)


if __name__ == "__main__":
    sys.exit(main())
