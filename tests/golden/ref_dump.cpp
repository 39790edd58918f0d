// Fixture dumper: drives the reference's own compiled filter / table / order
// code (linked from the objects oracle/Makefile builds out of the reference
// sources) through the same "-QorCandi C" sequence as
// matching/StudyPerformance.cpp:951-1600 split_C_test, and prints what the
// reference computes:
//
//   C <u> <n> <ids...>          candidate set of query vertex u (sorted)
//   T <a> <b> <nnz> <off...> | <adj...>   candidate-edge table T[a][b]
//   O <order...>                matching order
//   P <pivots...>               pivots (entry 0 unused)
//   M <bytes>                   computeMemoryCostInBytes
//
// Usage: ref_dump <data.txt> <query.txt> <GQL|CFL|NLF> <GQL|CFL>
// Only tests/golden/make_golden.py runs this, in the development container.
#include <cstdio>
#include <limits>
#include <string>

#include "graph/graph.h"
#include "matching/Args.h"
#include "matching/BuildTable.h"
#include "matching/EvaluateQuery.h"
#include "matching/FilterVertices.h"
#include "matching/GenerateFilteringPlan.h"
#include "matching/GenerateQueryPlan.h"
#include "matching/TaskPool.h"
#include "utility/splitGraph/SplitGraph.h"
#include "utility/statistics/intTimer.h"

int main(int argc, char** argv) {
    if (argc < 5) {
        fprintf(stderr, "usage: %s data query filter order\n", argv[0]);
        return 2;
    }
    std::string filter = argv[3], order = argv[4];
    Log::setLogFilePath("/tmp/psm_ref_dump.log");
    Graph* data = new Graph(true);
    data->loadGraphFromFile(argv[1]);
    Graph* query = new Graph(true);
    query->loadGraphFromFile(argv[2]);
    query->buildCoreTable();
    const ui qn = query->getVerticesCount();
    int64_t time_limit = intTimer::getClockNano() + (int64_t)3600 * 1000000000ll;
    FilterVertices::time_limit = time_limit;

    ui** cand = nullptr;
    ui* cnt = nullptr;
    ui* cfl_order = new ui[qn];
    TreeNode* cfl_tree = new TreeNode[qn];
    if (filter == "GQL")
        FilterVertices::GQLFilter(data, query, cand, cnt);
    else if (filter == "CFL")
        FilterVertices::CFLFilter(data, query, cand, cnt, cfl_order, cfl_tree);
    else
        FilterVertices::NLFFilter(data, query, cand, cnt);
    FilterVertices::sortCandidates(cand, cnt, qn);

    Edges*** em = new Edges**[qn];
    for (ui i = 0; i < qn; ++i) em[i] = new Edges*[qn];
    BuildTable::buildTables(data, query, cand, cnt, em);
    size_t mem = BuildTable::computeMemoryCostInBytes(query, cnt, em);

    for (ui u = 0; u < qn; ++u) {
        printf("C %u %u", u, cnt[u]);
        for (ui j = 0; j < cnt[u]; ++j) printf(" %u", cand[u][j]);
        printf("\n");
    }
    for (ui a = 0; a < qn; ++a)
        for (ui b = 0; b < qn; ++b) {
            if (!query->checkEdgeExistence(a, b)) continue;
            Edges* e = em[a][b];
            printf("T %u %u %u", a, b, e->edge_count_);
            for (ui i = 0; i <= e->vertex_count_; ++i) printf(" %u", e->offset_[i]);
            printf(" |");
            for (ui i = 0; i < e->edge_count_; ++i) printf(" %u", e->edge_[i]);
            printf("\n");
        }
    printf("M %zu\n", mem);

    TaskSlot::g_args = new GLOBALARGS(data, query, em, cand, cnt, std::numeric_limits<int64_t>::max(), time_limit);
    TaskSlot::g_args->engine_type = order == "GQL" ? "GQL" : "EXPLORE";
    SplitGraph* sg = new SplitGraph(data, query, JoinParadigm::LEFTDEEP, SplitPattern::SEED, SPLITMODE::NOSPLIT,
                                    time_limit);
    UnitArgs* ua = new UnitArgs(sg->getSubgraphs()[0], std::numeric_limits<int64_t>::max());
    ua->mapUidCandidates(TaskSlot::g_args);
    ua->mapUidEdgeMatrix(TaskSlot::g_args);
    Graph* unit = ua->query_graph->subgraph;
    if (order == "GQL") {
        GenerateQueryPlan::generateGQLQueryPlan(data, unit, ua);
    } else {
        GenerateFilteringPlan::generateCFLFilterPlan(data, ua);
        GenerateQueryPlan::generateCFLQueryPlan(unit, ua);
    }
    printf("O");
    for (ui i = 0; i < qn; ++i) printf(" %u", ua->order[i]);
    printf("\nP 0");
    for (ui i = 1; i < qn; ++i) printf(" %u", ua->pivots[i]);
    printf("\n");
    return 0;
}
