"""The Catch section walker that unfolds nested test sections into golden cases
(tests/golden/make_golden.py), on a synthetic snippet: each THEN leaf replays the statements of
its enclosing sections in order, a sibling's statements stay out, and a header that spans lines
still opens its section."""
import importlib.util
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SNIPPET = """SCENARIO("walk")
{
	GIVEN("a grid")
	{
		grid.track(pos1_idx);
		THEN("one")
		{
			CHECK(grid.list().size() == 1);
		}
		AND_WHEN("another")
		{
			grid.track(pos2_idx);
			THEN(
				"a header over"
				" two lines"
			) {
				CHECK(grid.list().size() == 2);
			}
		}
		AND_WHEN("reset") {
			grid.reset();
			THEN("empty") {
				CHECK(grid.list().size() == 0);
			}
		}
	}
}
"""


def _walker():
    spec = importlib.util.spec_from_file_location(
        "make_golden", os.path.join(ROOT, "tests", "golden", "make_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.catch_leaves


def test_leaves_replay_their_ancestors():
    lines = SNIPPET.split("\n")
    leaves = _walker()(lines, 1, len(lines))
    assert [lf["actions"] for lf in leaves] == [
        ["grid.track(pos1_idx);"],
        ["grid.track(pos1_idx);", "grid.track(pos2_idx);"],
        ["grid.track(pos1_idx);", "grid.reset();"],
    ]
    assert [lf["checks"] for lf in leaves] == [
        ["CHECK(grid.list().size() == 1);"],
        ["CHECK(grid.list().size() == 2);"],
        ["CHECK(grid.list().size() == 0);"],
    ]
