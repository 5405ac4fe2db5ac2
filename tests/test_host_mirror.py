"""The C++ host mirror (reverse-k-ranks_b200/host/B200Index.hpp) compiles inside the reference's
own header set -- the way a maintainer would add it to the query app -- against include/rkr.h."""
import os
import subprocess
import tempfile

import pytest

from checkers import reference_root

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(reference_root(), "src")

DRIVER = r'''
#include "util/VectorIO.hpp"
#include "util/TimeMemory.hpp"
#include "util/FileIO.hpp"
#include "struct/UserRankElement.hpp"
#include "struct/VectorMatrix.hpp"
#include "QS.hpp"
#include "QSRPNormalLP.hpp"
#include "US.hpp"
#include "B200Index.hpp"
using namespace ReverseMIPS;
int main(int argc, char **argv) {
    int n_item, n_query, n_user, dim;
    std::vector<VectorMatrix> data = readData(argv[1], argv[2], n_item, n_query, n_user, dim);
    std::unique_ptr<BaseIndex> index = B200::BuildIndex("QSRPNormalLP", data[1], data[0], argv[2], 20, 150, 40, argv[3]);
    std::vector<SingleQueryPerformance> perf(n_query);
    auto res = index->Retrieval(data[2], 10, n_query, perf);
    WriteRankResult(res, argv[2], "QSRPNormalLPB200", "top10");
    return 0;
}
'''


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference sources not present")
def test_b200_index_compiles_with_reference_headers():
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "rri_b200.cpp")
        open(src, "w").write(DRIVER)
        cmd = ["g++", "-std=c++17", "-fsyntax-only", "-fopenmp", "-w",
               "-I", os.path.join(ROOT, "oracle", "ref_shim"), "-I", os.path.join(REF, "include"),
               "-I", os.path.join(REF, "impl"), "-I", os.path.join(ROOT, "include"),
               "-I", os.path.join(ROOT, "reverse-k-ranks_b200", "host"), src]
        r = subprocess.run(cmd, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr[-3000:]
