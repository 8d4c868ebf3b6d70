"""Writes known_answers.json: the reference's own known-answer SQL tests for the aggregation path
(Warpstore tests/smoke.py:15-34), restated as table rows + the expected result rows.

The SQL table t(id INT, name VARCHAR, price DOUBLE, d DATE) is stored the engine's way: name as
dictionary codes (in insertion order: apple 0, banana 1, cherry 2, date 3), d as days since 1970-01-01.
Two table states are recorded: after the initial INSERT (smoke.py:17) and after the UPDATE / DELETE /
INSERT of smoke.py:23-28.  Expected values are the ones smoke.py asserts.
"""
import datetime
import json
import os

EPOCH = datetime.date(1970, 1, 1)


def days(s):
    return (datetime.date.fromisoformat(s) - EPOCH).days


state1 = {
    "id": [1, 2, 3, 4],
    "name": [0, 1, 2, 0],
    "price": [1.5, 0.25, 3.0, 2.5],
    "d": [days("2024-01-01"), days("2024-02-01"), days("2024-03-01"), days("2024-04-01")],
}
# UPDATE t SET price = price + 10 WHERE name = 'apple'; DELETE FROM t WHERE id = 2 (row 1 deleted);
# INSERT (5, 'date', 9.0, '2024-05-01')
state2 = {
    "id": [1, 2, 3, 4, 5],
    "name": [0, 1, 2, 0, 3],
    "price": [11.5, 0.25, 3.0, 12.5, 9.0],
    "d": [days("2024-01-01"), days("2024-02-01"), days("2024-03-01"), days("2024-04-01"), days("2024-05-01")],
    "deleted": [1],
}
cases = [
    {"name": "group by", "sql": "SELECT name, COUNT(*), SUM(price), MIN(d) FROM t GROUP BY name ORDER BY name",
     "state": 1, "expect": [[0, 2, 4.0, days("2024-01-01")], [1, 1, 0.25, days("2024-02-01")],
                            [2, 1, 3.0, days("2024-03-01")]], "source": "tests/smoke.py:20-21"},
    {"name": "or filter", "sql": "SELECT COUNT(*), SUM(price) FROM t WHERE name LIKE 'b%' OR price > 2",
     "state": 1, "expect": [[3, 5.75]], "source": "tests/smoke.py:22"},
    {"name": "having", "sql": "SELECT name, SUM(price) s FROM t GROUP BY name HAVING s > 5 ORDER BY s DESC",
     "state": 2, "expect": [[0, 24.0], [3, 9.0]], "source": "tests/smoke.py:31"},
    {"name": "case group",
     "sql": "SELECT CASE WHEN price > 10 THEN 1 ELSE 0 END AS big, COUNT(*) FROM t GROUP BY big ORDER BY big",
     "state": 2, "expect": [[0, 2], [1, 2]], "source": "tests/smoke.py:33"},
    {"name": "year()", "sql": "SELECT YEAR(d) y, COUNT(*) FROM t GROUP BY y ORDER BY y", "state": 2,
     "expect": [[2024, 4]], "source": "tests/smoke.py:34"},
]
out = {"states": {"1": state1, "2": state2}, "cases": cases}
path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "known_answers.json")
with open(path, "w") as f:
    json.dump(out, f, indent=1)
print(path)
