% two triangles sharing vertex 3; vertex ids 8..19 unused except 20
1 2
2 3
3 1
3 4
4 5
5 3
5 20
