"""The router patch recipe (baseline/patch_router.py) on a stand-in source with the sites it looks for.

The stand-in holds only the short fragments the recipe anchors on, in the functions that hold them in pcbroute's
src/router.cpp (rebuild_costs, refresh_costs, route_waves). Checked: each of the eight hook calls goes in once, after
its site and inside its function; a missing site or a duplicated wait condition stops the recipe instead of
producing a router without a hook. CPU only.
"""
import importlib.util
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _recipe():
    spec = importlib.util.spec_from_file_location("patch_router", os.path.join(ROOT, "baseline", "patch_router.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


STANDIN = """\
void rebuild_costs(float pres, bool hard) {
    std::vector<std::thread> th;
    for (auto& t : th) t.join();
}

void refresh_costs(size_t id, const std::vector<Span>& spans) {
    for (int c = 0; c < n; ++c) {
                if (kind) st(R.vcst[c], vcost_of(R, c));
                else st(R.cst[l][c], cost_of(R, l, c));
            }
}

void route() {
    auto route_waves = [&](const std::vector<int>& todo, float pres, bool hard) {
        const size_t n = order.size();
        auto worker = [&]() {
            cv.wait(lk, [&] {
                return (ready && (!anydep || dep[next] < int(cursor)));
            });
            saved[i] = {J.paths, J.keep, J.stubs, J.unrouted};
        };
        for (;;) {
                        if (fine) {
                            commits.push_back(std::move(blocks));
                        }
        }
        for (auto& t : th) t.join();
    };
}
"""


def test_each_hook_goes_in_once_at_its_site():
    m = _recipe()
    out = m.patch(STANDIN)
    for h in m.HOOKS:
        assert out.count(h + "(") == 1, h
    pos = {h: out.index(h + "(") for h in m.HOOKS}
    rebuild, refresh, waves = (out.index(f) for f in ("void rebuild_costs", "void refresh_costs", "auto route_waves"))
    assert rebuild < pos["pcbgh_rebuilt"] < refresh < pos["pcbgh_refreshed"] < waves
    # inside route_waves, in the order the worker meets them
    order = ["pcbgh_begin", "pcbgh_allow", "pcbgh_started", "pcbgh_verdict", "pcbgh_commit", "pcbgh_end"]
    assert waves < pos[order[0]] and [pos[h] for h in order] == sorted(pos[h] for h in order)
    # the wait condition keeps its own test and adds the scheduler's
    assert "(!anydep || dep[next] < int(cursor)) && pcbgh_allow(next, cursor, commits.size()));" in out
    # the verdict comes before the commit branch, the commit after the push
    assert out.index("pcbgh_verdict(") < out.index("if (fine) {")
    assert out.index("commits.push_back(std::move(blocks));") < pos["pcbgh_commit"]
    # nothing of the stand-in is lost
    assert out.replace("\n", "").count(";") >= STANDIN.replace("\n", "").count(";")


@pytest.mark.parametrize("site", ["const size_t n = order.size();\n",
                                  "saved[i] = {J.paths, J.keep, J.stubs, J.unrouted};\n",
                                  "                        if (fine) {\n",
                                  "else st(R.cst[l][c], cost_of(R, l, c));\n            }\n"])
def test_a_missing_site_stops_the_recipe(site):
    m = _recipe()
    assert site in STANDIN
    with pytest.raises(SystemExit):
        m.patch(STANDIN.replace(site, ""))


def test_a_duplicated_wait_condition_stops_the_recipe():
    m = _recipe()
    cond = "(!anydep || dep[next] < int(cursor)));"
    with pytest.raises(SystemExit):
        m.patch(STANDIN.replace("void route() {", "void other() { return (x && " + cond + " }\nvoid route() {"))
