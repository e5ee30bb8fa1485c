"""bench.py's GPU arm cannot run on the host; this checks statically that every name its functions read is defined
(a local, an argument, an import, a module-level name or a builtin), so that an edit cannot leave a line the GPU run
would only reach at its end."""
import ast
import builtins
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_bench_reads_no_undefined_name():
    tree = ast.parse(open(os.path.join(ROOT, "bench.py")).read())
    module = {n.name for n in tree.body if isinstance(n, (ast.FunctionDef, ast.ClassDef))}
    module |= {t.id for n in tree.body if isinstance(n, ast.Assign) for t in n.targets if isinstance(t, ast.Name)}
    module |= {(a.asname or a.name).split(".")[0] for n in tree.body if isinstance(n, (ast.Import, ast.ImportFrom))
               for a in n.names}
    module |= {"__file__", "__name__"}
    for fn in (n for n in tree.body if isinstance(n, ast.FunctionDef)):
        defined, used = set(), set()
        for node in ast.walk(fn):
            if isinstance(node, ast.Name):
                (defined if isinstance(node.ctx, (ast.Store, ast.Del)) else used).add(node.id)
            elif isinstance(node, (ast.FunctionDef, ast.ClassDef)):
                defined.add(node.name)
            elif isinstance(node, ast.arg):
                defined.add(node.arg)
            elif isinstance(node, ast.ExceptHandler) and node.name:
                defined.add(node.name)
            elif isinstance(node, (ast.Import, ast.ImportFrom)):
                defined |= {(a.asname or a.name).split(".")[0] for a in node.names}
        missing = sorted(u for u in used - defined - module if not hasattr(builtins, u))
        assert not missing, f"bench.py {fn.name}() reads undefined names {missing}"
