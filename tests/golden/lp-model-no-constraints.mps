NAME
OBJSENSE
 MAX
ROWS
 N  OBJ
COLUMNS
    x1        OBJ       1
RHS
RANGES
BOUNDS
 MI bounds    x1
 UP bounds    x1        1
ENDATA
