# K5 with repeated edges (both directions) and self-loops, 1-based
1 2
2 1
1 3
1 4
1 5
2 3
3 2
2 4
2 5
3 3
3 4
3 5
4 5
5 4
5 5
1 2
