% nothing but comments
# still nothing
