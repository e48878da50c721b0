"""Write a copy of pcbroute's src/router.cpp with the back end's hook calls added (baseline/router_hooks.h).

    python baseline/patch_router.py <pcbroute>/src/router.cpp <out>/router.cpp

A build recipe: it reads the router's source where it lies and writes the patched copy under baseline/_ref/ (git-
ignored); nothing of the router's source enters this repository. Each hook goes in at one site, found by a short
fragment of the line it follows or extends: the first occurrence after the opening line of the function that holds
the site (the worker's wait condition must occur exactly once in the file). The script stops with an error if a
site is not found, or if the result does not hold each of the eight hook calls exactly once, so a changed router
fails to build instead of building without a hook. The hooks read the router's state and change none of it (see
router_hooks.h).
"""
import sys

HOOKS = ("pcbgh_rebuilt", "pcbgh_refreshed", "pcbgh_begin", "pcbgh_allow", "pcbgh_started", "pcbgh_verdict",
         "pcbgh_commit", "pcbgh_end")


def insert_after(src, scope, anchor, text, start=0):
    """Insert `text` after the single occurrence of `anchor` inside the function that begins at `scope`."""
    a = src.index(scope, start) if scope else start
    k = src.find(anchor, a)
    if k < 0:
        raise SystemExit(f"patch_router: site not found after {scope!r}: {anchor!r}")
    k += len(anchor)
    return src[:k] + text + src[k:]


def patch(s):
    """The router source `s` with the hook calls added."""
    # mirror: every grid after a rebuild, the changed spans after a refresh
    s = insert_after(s, "void rebuild_costs(float pres, bool hard) {", "for (auto& t : th) t.join();\n",
                     "        pcbgh_rebuilt(rcs, hist, NL, G.nx, G.ny);\n")
    s = insert_after(s, "void refresh_costs(size_t id, const std::vector<Span>& spans) {",
                     "else st(R.cst[l][c], cost_of(R, l, c));\n            }\n",
                     "        pcbgh_refreshed(k, kind, l, spans);\n")
    # scheduler: route_waves
    rw = "auto route_waves = [&](const std::vector<int>& todo, float pres, bool hard) {"
    s = insert_after(s, rw, "const size_t n = order.size();\n", "            pcbgh_begin(order, jobs, G, o.window);\n")
    cond = "(!anydep || dep[next] < int(cursor))"
    i = s.index(rw)
    k = s.find(cond + ");", i)
    if k < 0 or s.count(cond + ");") != 1:
        raise SystemExit("patch_router: the worker's wait condition was not found exactly once")
    s = s[:k] + cond + " && pcbgh_allow(next, cursor, commits.size()));" + s[k + len(cond) + 2:]
    s = insert_after(s, rw, "saved[i] = {J.paths, J.keep, J.stubs, J.unrouted};\n",
                     "                        pcbgh_started(i, cursor, v0);\n")
    fine = "                        if (fine) {\n"
    k = s.find(fine, s.index(rw))
    if k < 0:
        raise SystemExit("patch_router: the commit check was not found")
    s = s[:k] + "                        pcbgh_verdict(cursor, fine, startver[cursor], commits, C.touch, C.touchv, BN * NL);\n" + s[k:]
    s = insert_after(s, rw, "commits.push_back(std::move(blocks));\n",
                     "                            pcbgh_commit(cursor, commits.size() - 1);\n")
    s = insert_after(s, rw, "for (auto& t : th) t.join();\n", "            pcbgh_end();\n")
    for h in HOOKS:
        if s.count(h + "(") != 1:
            raise SystemExit(f"patch_router: {h} is not called exactly once in the patched router")
    return s


def main():
    src_path, out_path = sys.argv[1], sys.argv[2]
    s = patch(open(src_path).read())
    with open(out_path, "w") as f:
        f.write(s)


if __name__ == "__main__":
    main()
